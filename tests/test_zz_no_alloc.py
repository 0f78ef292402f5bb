"""The allocation-free decimation entry point, hv_decimate_noalloc.

It exists for callers that cannot allocate device memory when they call it
(real-time audio threads, processes whose GPU memory is wholly held by a
caching allocator or a fixed budget): its scratch is a fixed array compiled
into the library. These tests call it through the C ABI and check that it
gives the decimated waveform the regular pipeline produces (hv_harvest_stages'
y) on two calls in a row, which also shows that the second call is unaffected
by what the first left in the shared scratch. The file is named to be
collected last."""
import ctypes as ct

import numpy as np
import pytest

import harvest_cuda_b200 as hv
from harvest_cuda_b200 import _native, signals


def _decimate_noalloc(x, fs):
    import torch
    ratio = min(12, max(1, int(fs / 8000.0 + 0.5)))
    x_dev = torch.from_numpy(np.ascontiguousarray(x)).to("cuda:0")
    y_dev = torch.full((-(-x.size // ratio),), np.nan, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    status = _native.lib.hv_decimate_noalloc(x_dev.data_ptr(), x.size, fs, 0, y_dev.data_ptr(), None)
    _native.raise_for(status)
    torch.cuda.synchronize()
    return y_dev.cpu().numpy()


@pytest.mark.gpu
def test_no_alloc_decimation_matches_pipeline_twice(gpu):
    cases = [(signals.kind_clip("speechlike", 1.7, 44100), 44100),
             (signals.glide_clip(2.3, 16000, seed=4)[0], 16000)]
    for x, fs in cases:   # two calls in a row, different rates and lengths
        got = _decimate_noalloc(x, fs)
        want = hv.api.stages(x, fs)["y"]
        assert got.shape == want.shape
        # The stage-parity tolerance of the decimated waveform.
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-12 * np.abs(want).max())


def test_no_alloc_rejects_input_beyond_its_scratch():
    status = _native.lib.hv_decimate_noalloc(None, (1 << 20) + 1, 16000, 0, None, None)
    assert status == _native.HV_INVALID_ARGUMENT
    assert "at most 1048576 samples" in _native.last_error()
