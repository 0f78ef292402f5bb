"""The allocation-free decimation entry point, hv_decimate_noalloc.

It exists for callers that cannot allocate device memory when they call it
(real-time audio threads that must not block in the driver's allocator,
processes whose GPU memory is wholly held by a caching allocator or a fixed
budget): its scratch is a fixed array compiled into the library, so input is
limited to 1,048,576 samples per call. These tests call it through the C ABI
and check that it gives the decimated, DC-free waveform that the regular
pipeline produces (hv_harvest_stages' y) and that the CPU checker produces,
on calls in a row over different rates and lengths (each call overwrites
what the previous one left in the shared scratch), at the size limit for the
two largest decimation lags, at 8 kHz (no decimation, a plain copy), and on
a side stream. The file is named to be collected last."""
import numpy as np
import pytest

import harvest_cuda_b200 as hv
from harvest_cuda_b200 import _native, signals

LIMIT = 1 << 20


def _decimate_noalloc(x, fs, stream=None):
    import torch
    ratio = min(12, max(1, int(fs / 8000.0 + 0.5)))
    x_dev = torch.from_numpy(np.ascontiguousarray(x)).to("cuda:0")
    y_dev = torch.full((-(-x.size // ratio),), np.nan, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    handle = None if stream is None else stream.cuda_stream
    status = _native.lib.hv_decimate_noalloc(x_dev.data_ptr(), x.size, fs, 0, y_dev.data_ptr(), handle)
    _native.raise_for(status)
    torch.cuda.synchronize()
    return y_dev.cpu().numpy()


def _close(got, want):
    # The stage-parity tolerance of the decimated waveform.
    assert got.shape == want.shape
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12 * np.abs(want).max())


def _long_clip(fs, seconds):
    x, _ = signals.glide_clip(seconds, fs, seed=fs)
    x = np.resize(x, LIMIT)   # exactly at the limit
    return np.ascontiguousarray(x)


@pytest.mark.gpu
def test_no_alloc_decimation_matches_pipeline_and_checker(gpu, checker):
    cases = [(signals.kind_clip("speechlike", 1.7, 44100), 44100),   # ratio 6
             (signals.glide_clip(2.3, 16000, seed=4)[0], 16000),      # ratio 2
             (signals.kind_clip("high", 0.9, 8000), 8000),            # ratio 1: a copy
             (_long_clip(48000, 22.0), 48000),                        # limit, ratio 6, lag 144
             (_long_clip(96000, 11.0), 96000)]                        # limit, ratio 12, lag 144
    for x, fs in cases:   # calls in a row: each follows a call of another rate and length
        got = _decimate_noalloc(x, fs)
        assert np.all(np.isfinite(got))
        _close(got, hv.api.stages(x, fs)["y"])
        _close(got, checker.stages(x, fs)["y"])


@pytest.mark.gpu
def test_no_alloc_repeat_and_side_stream(gpu):
    import torch
    x, _ = signals.glide_clip(3.1, 24000, seed=9)
    first = _decimate_noalloc(x, 24000)
    other = _decimate_noalloc(signals.kind_clip("noise", 0.5, 192000), 192000)
    assert np.all(np.isfinite(other))
    second = _decimate_noalloc(x, 24000)
    np.testing.assert_array_equal(first, second)
    side = torch.cuda.Stream()
    on_side = _decimate_noalloc(x, 24000, stream=side)
    np.testing.assert_array_equal(first, on_side)


def test_no_alloc_rejects_input_beyond_its_scratch():
    status = _native.lib.hv_decimate_noalloc(None, LIMIT + 1, 16000, 0, None, None)
    assert status == _native.HV_INVALID_ARGUMENT
    assert "at most 1048576 samples" in _native.last_error()
