"""Parity with the reference's own CUDA path (its src/cuda_backend.cu and
src/engine.cpp, built by oracle/Makefile into oracle/_ref/libref_cuda.so), a
second reference beside its bundled WORLD: on the same clips the engine and
the reference's GPU build must meet the acceptance bar against each other
(time axis bit-exact, voicing agreement on >= 99.9 % of frames, voiced F0
within 1e-6 relative)."""
import numpy as np
import pytest

import harvest_cuda_b200 as hv
import oracle
from harvest_cuda_b200 import signals
from tests.test_gpu_parity import assert_parity

pytestmark = pytest.mark.gpu

CASES = [
    ("glide3s_16k", lambda: signals.glide_clip(3.0, 16000, seed=1)[0], 16000, 71.0, 800.0, 5.0),
    ("glide2s_16k_wide", lambda: signals.glide_clip(2.0, 16000, seed=2)[0], 16000, 50.0, 1100.0, 5.0),
    ("segmented8s_44k", lambda: signals.segmented_clip(8.0, 44100, seed=3), 44100, 71.0, 800.0, 5.0),
    ("speech48k_1ms", lambda: signals.kind_clip("speechlike", 1.5, 48000), 48000, 71.0, 800.0, 1.0),
    ("short8k", lambda: signals.kind_clip("high", 0.4, 8000), 8000, 71.0, 800.0, 5.0),
]


@pytest.fixture(scope="module")
def reference_gpu(gpu):
    r = oracle.reference_cuda()
    if r is None:
        pytest.skip("the reference's CUDA build (oracle/_ref/libref_cuda.so) is absent")
    if not r.available(0):
        pytest.skip("the reference's CUDA build does not run on this device")
    return r


@pytest.mark.parametrize("name,make,fs,floor,ceil,period", CASES, ids=[c[0] for c in CASES])
def test_engine_matches_reference_cuda(reference_gpu, name, make, fs, floor, ceil, period):
    x = make()
    expected = reference_gpu.harvest(x, fs, floor, ceil, period)
    actual = hv.harvest(x, fs, floor, ceil, period)
    m = assert_parity(actual, expected)
    if name != "short8k":
        assert m["joint_voiced_frames"] > 0
