"""Boundary tests that need no GPU: the C ABI library loads and exports
exactly what include/harvest_b200.h declares, and the Python API rejects bad
arguments with the reference's exception classes
(reference tests/test_compatibility.py:60-99, 137-143)."""
import os
import re
import subprocess

import numpy as np
import pytest

import harvest_cuda_b200 as hv
from harvest_cuda_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fname in os.listdir(os.path.join(ROOT, "include")):
        if fname.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fname)).read()
            names |= set(re.findall(r"HV_API\s+[\w\s\*]+?\b(hv_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    declared = _declared()
    assert declared, "no declarations found"
    out = subprocess.run(["nm", "-D", "--defined-only", _native.LIBRARY_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (hv_\w+)", out))
    assert declared == exported
    assert declared == set(_native.SIGNATURES)
    for name in declared:
        assert getattr(_native.lib, name) is not None


def test_library_has_no_driver_link_dependency():
    # Loads on machines without a GPU driver: libcuda is resolved at run time.
    out = subprocess.run(["ldd", _native.LIBRARY_PATH], capture_output=True, text=True).stdout
    assert "libcuda.so" not in out


@pytest.mark.parametrize("kwargs", [
    {"fs": 0}, {"fs": 7999}, {"fs": 192001}, {"f0_floor": 0}, {"f0_floor": 800},
    {"f0_ceil": float("inf")}, {"f0_ceil": 5000}, {"frame_period": 0},
    {"frame_period": float("nan")}, {"frame_period": -1.0},
])
def test_invalid_parameters(kwargs):
    params = {"fs": 24000, **kwargs}
    with pytest.raises(ValueError):
        hv.harvest(np.zeros(2400), **params)


@pytest.mark.parametrize("x", [np.zeros(0), np.array([np.nan, 0.0, 0, 0, 0, 0]),
                               np.array([np.inf, 0.0, 0, 0, 0, 0]), np.zeros(5)])
def test_invalid_samples(x):
    with pytest.raises(ValueError):
        hv.harvest(x, 24000)


@pytest.mark.parametrize("x", [np.zeros(100, dtype=np.float32), np.zeros((2, 100)),
                               np.zeros(100)[::2], [0.0] * 100])
def test_rejects_wrong_array_type(x):
    with pytest.raises(TypeError):
        hv.harvest(x, 24000)


def test_device_argument_validation():
    x = np.zeros(2400)
    assert not hv.cuda_available(device=-1)
    with pytest.raises(ValueError, match="nonnegative"):
        hv.harvest(x, 24000, device=-1)
    with pytest.raises(TypeError):
        hv.harvest(x, 24000, 71.0, 800.0, 5.0, 0)
    with pytest.raises(TypeError):
        hv.harvest(x, 24000, device="cuda:0")


def test_gpu_required():
    if hv.cuda_available():
        pytest.skip("GPU available")
    with pytest.raises(RuntimeError):
        hv.harvest(np.zeros(2400), 24000)
    with pytest.raises(RuntimeError):
        hv.harvest_many([np.zeros(2400), np.zeros(4800)], 24000)


def test_clear_empty_cache():
    hv.clear_cache()
    hv.clear_cache()


def test_output_length_matches_checker():
    import oracle
    for n, fs, period in [(48000, 16000, 5.0), (2646000, 44100, 5.0), (6, 24000, 5.0),
                          (12345, 11025, 7.3), (96000, 48000, 1.0)]:
        assert hv.output_length(n, fs, period) == oracle.port().lib.oracle_output_length(n, fs, period)


def test_batch_argument_validation():
    x = np.zeros(4800)
    with pytest.raises(ValueError):
        hv.harvest_batch(x, [0, 2400, 2400], 24000)   # empty clip
    with pytest.raises(ValueError):
        hv.harvest_batch(x, [0, 5000], 24000)          # beyond x
    with pytest.raises(ValueError):
        hv.harvest_batch(x, [0], 24000)
    with pytest.raises(TypeError):
        hv.harvest_batch(x.astype(np.float32), [0, 4800], 24000)


def test_batch_pipeline_validates_arguments_before_needing_a_gpu():
    from harvest_cuda_b200.pipeline import BatchPipeline
    with pytest.raises(TypeError):
        BatchPipeline(16000.0)
    with pytest.raises(ValueError):
        BatchPipeline(16000, depth=1)
    import torch
    if not torch.cuda.is_available():
        with pytest.raises(RuntimeError, match="CUDA"):
            BatchPipeline(16000)
