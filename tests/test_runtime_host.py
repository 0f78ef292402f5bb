"""Host fault injection for the engine's runtime (device check, contexts,
growing device buffers and the per-device workspace cache), compiled with
g++ against fake CUDA headers whose calls fail on demand: see
tests/cpp/test_runtime.cpp. Needs no GPU and no CUDA toolkit."""
import os
import shutil
import subprocess

import pytest

CPP = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cpp")
BINARY = os.path.join(CPP, "_build", "test_runtime")


@pytest.fixture(scope="module")
def runtime_test():
    if shutil.which("g++") is None or shutil.which("make") is None:
        pytest.skip("g++ and make are needed to build the host runtime test")
    out = subprocess.run(["make", "-s", "-C", CPP], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    return BINARY


@pytest.mark.parametrize("mode", [[], ["no-driver"]], ids=["all", "no-driver"])
def test_runtime_fault_injection(runtime_test, mode):
    out = subprocess.run([runtime_test, *mode], capture_output=True, text=True, timeout=180)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "passed" in out.stdout
