"""The device-resident API (harvest_cuda_b200.device): CUDA tensors or
__dlpack__ arrays in, CUDA tensors out, ordered on the caller's current
PyTorch stream. Results must equal the NumPy API's bit for bit."""
import numpy as np
import pytest

import harvest_cuda_b200 as hv
from harvest_cuda_b200 import device, signals

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _clips():
    return [signals.glide_clip(s, 16000, seed=i)[0] for i, s in enumerate((1.2, 0.6, 2.1))]


def test_batch_matches_numpy_api_on_default_and_side_streams(gpu):
    torch = _torch()
    clips = _clips()
    packed, offsets = signals.pack(clips)
    want_f0, want_t, want_off = hv.harvest_batch(packed, offsets, 16000, 50.0, 1100.0, 5.0)
    # Default stream: the input is written by a copy on that stream just
    # before the call, so the engine must order its work after it.
    x = torch.zeros(packed.size, dtype=torch.float64, device="cuda")
    x.copy_(torch.from_numpy(packed).cuda())
    f0, t, off = device.harvest_batch(x, offsets, 16000, 50.0, 1100.0, 5.0)
    assert np.array_equal(off, want_off)
    assert np.array_equal(f0.cpu().numpy(), want_f0) and np.array_equal(t.cpu().numpy(), want_t)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        y = torch.from_numpy(packed).cuda()
        f0, t, _ = device.harvest_batch(y, offsets, 16000, 50.0, 1100.0, 5.0, check_finite=False)
        got = f0.cpu().numpy()
    assert np.array_equal(got, want_f0)


def test_single_clip_and_dlpack_input(gpu):
    torch = _torch()
    x = signals.glide_clip(1.5, 24000, seed=9)[0]
    want = hv.harvest(x, 24000)

    class Foreign:      # an array known to us only through the DLPack protocol
        def __init__(self, t):
            self.t = t

        def __dlpack__(self, **kw):
            return self.t.__dlpack__(**kw)

        def __dlpack_device__(self):
            return self.t.__dlpack_device__()

    f0, t = device.harvest(Foreign(torch.from_numpy(x).cuda()), 24000)
    assert np.array_equal(f0.cpu().numpy(), want[0]) and np.array_equal(t.cpu().numpy(), want[1])


def test_rejects_non_finite_and_bad_arguments(gpu):
    torch = _torch()
    x = torch.from_numpy(signals.glide_clip(0.5, 16000)[0].copy()).cuda()
    x[100] = float("nan")
    with pytest.raises(ValueError, match="finite"):
        device.harvest(x, 16000)
    with pytest.raises(TypeError):
        device.harvest(x.float(), 16000)
    with pytest.raises(ValueError):
        device.harvest_batch(x, [0, x.numel() + 1], 16000)


def test_pcm16_batch_equals_converted_float_input(gpu):
    torch = _torch()
    clips = [np.clip(np.round(c * 32768 * 2), -32768, 32767).astype(np.int16)
             for c in (signals.glide_clip(s, 16000, seed=i)[0] for i, s in enumerate((1.0, 2.5, 0.4)))]
    pcm = np.concatenate(clips)
    offsets = np.concatenate([[0], np.cumsum([len(c) for c in clips])]).astype(np.int64)
    want = hv.harvest_batch(pcm.astype(np.float64) / 32768.0, offsets, 16000)
    got = hv.harvest_batch_pcm16(pcm, offsets, 16000)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    # Device PCM16 input through the C ABI.
    import ctypes as ct
    from harvest_cuda_b200 import _native
    x = torch.from_numpy(pcm).cuda()
    f0 = torch.empty(int(want[2][-1]), dtype=torch.float64, device="cuda")
    status = _native.lib.hv_harvest_batch_pcm16(
        x.data_ptr(), offsets.ctypes.data_as(ct.POINTER(ct.c_int64)), len(clips), 16000, 71.0, 800.0, 5.0, 0,
        f0.data_ptr(), None, _native.HV_DEVICE_POINTERS | _native.HV_NULL_IS_LEGACY_STREAM, None)
    _native.raise_for(status)
    assert np.array_equal(f0.cpu().numpy(), want[0])
