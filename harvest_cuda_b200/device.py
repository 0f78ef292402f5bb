"""Harvest on device-resident arrays (PyTorch CUDA tensors, or any CUDA array
exposing ``__dlpack__``, taken without a copy).

For pipelines whose audio already lives on the GPU (training data loaders,
batched evaluation): no host round trip, and the work is ordered on the
caller's current PyTorch stream, so the call returns as soon as it is
enqueued. Results are float64 CUDA tensors on the input's device.

* ``harvest(x, fs, ...)``: one clip, ``(f0, times)``.
* ``harvest_batch(x, offsets, fs, ...)``: clips packed back to back,
  ``(f0, times, out_offsets)`` packed the same way.

The differentiable variant is ``harvest_cuda_b200.autograd.harvest_f0``.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch

from . import _native

__all__ = ["harvest", "harvest_batch"]


def _as_tensor(x):
    if not torch.is_tensor(x):
        if not hasattr(x, "__dlpack__"):
            raise TypeError("x must be a CUDA tensor or an array exposing __dlpack__")
        x = torch.from_dlpack(x)
    if x.dtype != torch.float64 or x.dim() != 1 or not x.is_cuda:
        raise TypeError("x must be a 1-D float64 CUDA array")
    return x.contiguous()


def harvest_batch(x, offsets, fs, f0_floor=71.0, f0_ceil=800.0, frame_period=5.0, *, graph=True,
                  check_finite=True):
    """Harvest on clips packed back to back in the 1-D float64 CUDA array
    ``x``; clip c is ``x[offsets[c]:offsets[c+1]]`` (``offsets``: host
    sequence of ``clips + 1`` ints). Returns ``(f0, times, out_offsets)``
    with ``f0`` and ``times`` float64 CUDA tensors and ``out_offsets`` a
    NumPy int64 array. With ``check_finite`` (one device-to-host read), a
    non-finite sample raises ``ValueError`` as the NumPy API does; without
    it the call never waits for the GPU."""
    x = _as_tensor(x)
    offs = np.ascontiguousarray(offsets, dtype=np.int64)
    if offs.ndim != 1 or offs.size < 2 or offs[0] < 0 or offs[-1] > x.numel() or np.any(np.diff(offs) < 0):
        raise ValueError("offsets must hold clips + 1 nondecreasing entries within x")
    fs, period = int(fs), float(frame_period)
    counts = [_native.lib.hv_output_length(int(b - a), fs, period) for a, b in zip(offs[:-1], offs[1:])]
    if min(counts) < 0:
        raise ValueError("invalid length, sampling rate or frame period")
    out_offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    if check_finite and not bool(torch.isfinite(x[offs[0]:offs[-1]]).all()):
        raise ValueError("x must contain only finite samples")
    f0 = torch.empty(int(out_offsets[-1]), dtype=torch.float64, device=x.device)
    times = torch.empty_like(f0)
    flags = _native.HV_DEVICE_POINTERS | _native.HV_NULL_IS_LEGACY_STREAM
    if not graph:
        flags |= _native.HV_NO_GRAPH
    stream = torch.cuda.current_stream(x.device).cuda_stream
    status = _native.lib.hv_harvest_batch(
        x.data_ptr(), offs.ctypes.data_as(ct.POINTER(ct.c_int64)), offs.size - 1, fs, float(f0_floor),
        float(f0_ceil), period, x.device.index, f0.data_ptr(), times.data_ptr(), flags,
        ct.c_void_p(stream or None))
    _native.raise_for(status)
    return f0, times, out_offsets


def harvest(x, fs, f0_floor=71.0, f0_ceil=800.0, frame_period=5.0, *, check_finite=True):
    """One clip on the device: ``(f0, times)`` as float64 CUDA tensors."""
    x = _as_tensor(x)
    f0, times, _ = harvest_batch(x, [0, x.numel()], fs, f0_floor, f0_ceil, frame_period,
                                 graph=False, check_finite=check_finite)
    return f0, times
