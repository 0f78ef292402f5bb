"""Differentiable Harvest: F0 with a gradient with respect to the waveform.

Harvest's F0 is piecewise smooth in the waveform. Its discrete choices
(which candidates survive, voicing, FixF0Contour's extensions and merges,
the smoothing sections) are held fixed as recorded by the forward pass;
within that region every output F0 is a smooth function of the waveform
through

* the refined candidate it copies: FixF0's weighted mean of instantaneous
  frequencies at up to six harmonic bins of a Blackman-windowed spectrum of
  the decimated waveform (reference harvest.cpp:507-536 in its bundled
  WORLD), or FixStep4's linear fill between two such values;
* the zero-phase Butterworth smoothing of its voiced section and the
  resampling to ``frame_period``;
* the decimation and DC removal that produce the internal waveform.

The backward pass (``hv_harvest_grad_backward``) runs the transposes of
these maps on the GPU, recomputing the spectra from the waveform instead of
storing them. Frames whose F0 is 0 (unvoiced) have zero gradient. Across a
discrete switch, such as a candidate crossing a threshold or a window length
changing, the F0 jumps and no derivative exists; the gradient is that of the
smooth piece the forward pass fell in.
"""
from __future__ import annotations

import ctypes as ct

import torch

from . import _native

__all__ = ["HarvestF0", "harvest_f0", "RawCandidates", "raw_candidates"]


def _settings(fs, f0_floor, f0_ceil, frame_period):
    return int(fs), float(f0_floor), float(f0_ceil), float(frame_period)


def _frames(offsets, fs, period):
    """Per-clip frame counts at `period` ms, as the engine computes them."""
    out = []
    for a, b in zip(offsets[:-1], offsets[1:]):
        n = _native.lib.hv_output_length(b - a, fs, period)
        if n < 0:
            raise ValueError("invalid length, sampling rate or frame period")
        out.append(int(n))
    return out


def _stream(device):
    return ct.c_void_p(torch.cuda.current_stream(device).cuda_stream or None)


class HarvestF0(torch.autograd.Function):
    """``HarvestF0.apply(x, offsets, fs, f0_floor, f0_ceil, frame_period)``.

    ``x`` is a 1-D float64 CUDA tensor holding clips packed back to back,
    ``offsets`` a tuple of ``clips + 1`` ints (``offsets[0] == 0``,
    ``offsets[-1] == x.numel()``). Returns the packed F0 of every clip
    (frames of ``frame_period`` ms, clips in order) and its time axis; only
    the F0 carries a gradient, to ``x``."""

    @staticmethod
    def forward(ctx, x, offsets, fs, f0_floor, f0_ceil, frame_period):
        fs, f0_floor, f0_ceil, frame_period = _settings(fs, f0_floor, f0_ceil, frame_period)
        if x.dtype != torch.float64 or x.dim() != 1 or not x.is_cuda:
            raise TypeError("x must be a 1-D float64 CUDA tensor")
        offsets = tuple(int(o) for o in offsets)
        if len(offsets) < 2 or offsets[0] != 0 or offsets[-1] != x.numel():
            raise ValueError("offsets must start at 0 and end at x.numel()")
        x = x.contiguous()
        if not bool(torch.isfinite(x).all()):
            raise ValueError("x must contain only finite samples")
        device = x.device.index if x.device.index is not None else torch.cuda.current_device()
        clips = len(offsets) - 1
        out_len = sum(_frames(offsets, fs, frame_period))
        tape_len = 2 * sum(_frames(offsets, fs, 1.0))
        f0 = torch.empty(out_len, dtype=torch.float64, device=x.device)
        times = torch.empty_like(f0)
        tape = torch.empty(tape_len, dtype=torch.float64, device=x.device)
        offs = (ct.c_int64 * len(offsets))(*offsets)
        status = _native.lib.hv_harvest_grad_forward(
            x.data_ptr(), offs, clips, fs, f0_floor, f0_ceil, frame_period, device,
            f0.data_ptr(), times.data_ptr(), tape.data_ptr(), _stream(x.device))
        _native.raise_for(status)
        ctx.save_for_backward(x, tape)
        ctx.args = (offsets, fs, f0_floor, f0_ceil, frame_period, device)
        ctx.mark_non_differentiable(times)
        return f0, times

    @staticmethod
    def backward(ctx, grad_f0, grad_times):
        x, tape = ctx.saved_tensors
        offsets, fs, f0_floor, f0_ceil, frame_period, device = ctx.args
        grad_x = None
        if ctx.needs_input_grad[0]:
            grad_f0 = grad_f0.to(torch.float64).contiguous()
            grad_x = torch.empty_like(x)
            offs = (ct.c_int64 * len(offsets))(*offsets)
            status = _native.lib.hv_harvest_grad_backward(
                x.data_ptr(), offs, len(offsets) - 1, fs, f0_floor, f0_ceil, frame_period, device,
                tape.data_ptr(), grad_f0.data_ptr(), grad_x.data_ptr(), _stream(x.device))
            _native.raise_for(status)
        return grad_x, None, None, None, None, None


def harvest_f0(x, fs, f0_floor=71.0, f0_ceil=800.0, frame_period=5.0):
    """Differentiable Harvest on one clip or a list of clips.

    ``x`` is a 1-D float64 CUDA tensor, or a list of them (run as one ragged
    batch). Returns ``(f0, times)`` for one clip, or a list of such pairs;
    ``f0`` is differentiable with respect to the clip samples."""
    single = torch.is_tensor(x)
    clips = [x] if single else list(x)
    if not clips:
        raise ValueError("no clips")
    offsets = [0]
    for c in clips:
        if not torch.is_tensor(c) or c.dim() != 1:
            raise TypeError("each clip must be a 1-D float64 CUDA tensor")
        offsets.append(offsets[-1] + c.numel())
    packed = clips[0] if single else torch.cat(clips)
    f0, times = HarvestF0.apply(packed, tuple(offsets), fs, f0_floor, f0_ceil, frame_period)
    if single:
        return f0, times
    counts = _frames(offsets, int(fs), float(frame_period))
    return list(zip(torch.split(f0, counts), torch.split(times, counts)))


class RawCandidates(torch.autograd.Function):
    """``RawCandidates.apply(x, offsets, fs, f0_floor, f0_ceil)``: the band-pass
    bank's per-band F0 candidates (WORLD's GetF0CandidateContour) of clips
    packed in ``x`` as for ``HarvestF0``, as a ``(bands, frames)`` float64 CUDA
    tensor (1 ms frames of all clips in order; 0 where a band has no
    candidate). Differentiable with respect to ``x``: the fine positions of
    the zero crossings and extrema move smoothly with the waveform, while the
    events themselves, each frame's interpolation segments and the range
    checks are held fixed. The backward pass runs the adjoint of the
    band-pass bank, the interval detectors and the decimation on the GPU."""

    @staticmethod
    def forward(ctx, x, offsets, fs, f0_floor, f0_ceil):
        fs, f0_floor, f0_ceil = int(fs), float(f0_floor), float(f0_ceil)
        if x.dtype != torch.float64 or x.dim() != 1 or not x.is_cuda:
            raise TypeError("x must be a 1-D float64 CUDA tensor")
        offsets = tuple(int(o) for o in offsets)
        if len(offsets) < 2 or offsets[0] != 0 or offsets[-1] != x.numel():
            raise ValueError("offsets must start at 0 and end at x.numel()")
        x = x.contiguous()
        if not bool(torch.isfinite(x).all()):
            raise ValueError("x must contain only finite samples")
        device = x.device.index if x.device.index is not None else torch.cuda.current_device()
        bands = int(_native.lib.hv_band_count(f0_floor, f0_ceil))
        if bands < 1:
            raise ValueError("invalid f0_floor/f0_ceil")
        frames = sum(_frames(offsets, fs, 1.0))
        raw = torch.empty((bands, frames), dtype=torch.float64, device=x.device)
        offs = (ct.c_int64 * len(offsets))(*offsets)
        _native.raise_for(_native.lib.hv_raw_candidates(
            x.data_ptr(), offs, len(offsets) - 1, fs, f0_floor, f0_ceil, device, raw.data_ptr(),
            _stream(x.device)))
        ctx.save_for_backward(x)
        ctx.args = (offsets, fs, f0_floor, f0_ceil, device)
        return raw

    @staticmethod
    def backward(ctx, grad_raw):
        (x,) = ctx.saved_tensors
        offsets, fs, f0_floor, f0_ceil, device = ctx.args
        grad_x = None
        if ctx.needs_input_grad[0]:
            grad_raw = grad_raw.to(torch.float64).contiguous()
            grad_x = torch.empty_like(x)
            offs = (ct.c_int64 * len(offsets))(*offsets)
            _native.raise_for(_native.lib.hv_raw_candidates_backward(
                x.data_ptr(), offs, len(offsets) - 1, fs, f0_floor, f0_ceil, device, grad_raw.data_ptr(),
                grad_x.data_ptr(), _stream(x.device)))
        return grad_x, None, None, None, None


def raw_candidates(x, fs, f0_floor=71.0, f0_ceil=800.0):
    """Differentiable per-band candidates of one clip (a ``(bands, frames)``
    tensor) or of a list of clips (a list of such tensors, run as one batch)."""
    single = torch.is_tensor(x)
    clips = [x] if single else list(x)
    if not clips:
        raise ValueError("no clips")
    offsets = [0]
    for c in clips:
        if not torch.is_tensor(c) or c.dim() != 1:
            raise TypeError("each clip must be a 1-D float64 CUDA tensor")
        offsets.append(offsets[-1] + c.numel())
    packed = clips[0] if single else torch.cat(clips)
    raw = RawCandidates.apply(packed, tuple(offsets), fs, f0_floor, f0_ceil)
    if single:
        return raw
    return list(torch.split(raw, _frames(offsets, int(fs), 1.0), dim=1))
