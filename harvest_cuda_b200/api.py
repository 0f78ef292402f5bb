"""The pyworld-compatible NumPy API of the engine.

``harvest``, ``cuda_available`` and ``clear_cache`` keep the reference
package's names, defaults, argument rules and exception classes
(reference python/harvest_cuda/__init__.py:24-43, src/bindings.cpp:60-80):

* ``x`` must be a 1-D, C-contiguous float64 NumPy array (read-only arrays are
  accepted); anything else raises ``TypeError``, as nanobind's
  ``ndarray<const double, numpy, ndim<1>, c_contig>.noconvert()`` does;
* ``device`` is keyword-only and must be an ``int``;
* invalid values raise ``ValueError``, a missing or unusable GPU raises
  ``RuntimeError``.

``harvest_batch`` and ``harvest_many`` add the ragged batched path, which
the reference does not have.
"""
from __future__ import annotations

import ctypes as ct
import operator

import numpy as np

from . import _native

__all__ = ["harvest", "harvest_batch", "harvest_batch_pcm16", "harvest_many", "cuda_available",
           "clear_cache", "output_length", "profile"]

_D = ct.POINTER(ct.c_double)


def _as_int(value, name):
    if isinstance(value, bool) or isinstance(value, float):
        raise TypeError(f"{name} must be an int, not {type(value).__name__}")
    try:
        return operator.index(value)
    except TypeError:
        raise TypeError(f"{name} must be an int, not {type(value).__name__}") from None


def _as_float(value, name):
    if isinstance(value, (str, bytes)) or value is None:
        raise TypeError(f"{name} must be a float, not {type(value).__name__}")
    try:
        return float(value)
    except (TypeError, ValueError):
        raise TypeError(f"{name} must be a float, not {type(value).__name__}") from None


def _check_array(x):
    if not isinstance(x, np.ndarray):
        raise TypeError(f"x must be a numpy.ndarray of float64, not {type(x).__name__}")
    if x.dtype != np.float64:
        raise TypeError(f"x must have dtype float64, not {x.dtype}")
    if x.ndim != 1:
        raise TypeError(f"x must be one-dimensional, not {x.ndim}-D")
    if not x.flags.c_contiguous:
        raise TypeError("x must be C-contiguous")
    return x


def cuda_available(device=0) -> bool:
    """Whether ``device`` is a visible GPU this engine supports (sm_100)."""
    device = _as_int(device, "device")
    return bool(_native.lib.hv_cuda_available(device))


def clear_cache() -> None:
    """Release cached GPU working memory on every device. Calls in flight
    keep their workspace until they finish."""
    _native.raise_for(_native.lib.hv_clear_cache())


def output_length(n, fs, frame_period=5.0) -> int:
    """Number of frames ``harvest`` returns for ``n`` samples."""
    out = _native.lib.hv_output_length(int(n), int(fs), float(frame_period))
    if out < 0:
        raise ValueError("invalid length, sampling rate or frame period")
    return int(out)


def harvest(x, fs, f0_floor=71.0, f0_ceil=800.0, frame_period=5.0, *, device=0):
    """Estimate F0 with Harvest on the GPU.

    x: contiguous 1-D float64 NumPy array; returns ``(f0, times)`` as new
    float64 arrays. ``device`` indexes the GPUs visible through
    CUDA_VISIBLE_DEVICES.
    """
    x = _check_array(x)
    fs = _as_int(fs, "fs")
    f0_floor = _as_float(f0_floor, "f0_floor")
    f0_ceil = _as_float(f0_ceil, "f0_ceil")
    frame_period = _as_float(frame_period, "frame_period")
    device = _as_int(device, "device")
    lib = _native.lib
    # Validate first so errors match the reference even for empty input.
    status = lib.hv_validate(x.ctypes.data_as(_D), x.size, fs, f0_floor, f0_ceil, frame_period)
    _native.raise_for(status)
    n = lib.hv_output_length(x.size, fs, frame_period)
    f0 = np.empty(n)
    times = np.empty(n)
    status = lib.hv_harvest(x.ctypes.data_as(_D), x.size, fs, f0_floor, f0_ceil, frame_period,
                            device, f0.ctypes.data_as(_D), times.ctypes.data_as(_D), n)
    _native.raise_for(status)
    return f0, times


def profile(x, fs, f0_floor=71.0, f0_ceil=800.0, frame_period=5.0, *, device=0):
    """``harvest`` plus a dict of per-stage device milliseconds."""
    x = _check_array(x)
    fs = _as_int(fs, "fs")
    device = _as_int(device, "device")
    lib = _native.lib
    _native.raise_for(lib.hv_validate(x.ctypes.data_as(_D), x.size, fs, float(f0_floor),
                                      float(f0_ceil), float(frame_period)))
    n = lib.hv_output_length(x.size, fs, float(frame_period))
    f0, times = np.empty(n), np.empty(n)
    stages = np.zeros(_native.HV_STAGE_COUNT)
    status = lib.hv_profile(x.ctypes.data_as(_D), x.size, fs, float(f0_floor), float(f0_ceil),
                            float(frame_period), device, f0.ctypes.data_as(_D),
                            times.ctypes.data_as(_D), n, stages.ctypes.data_as(_D))
    _native.raise_for(status)
    names = [lib.hv_stage_name(i).decode() for i in range(_native.HV_STAGE_COUNT)]
    return f0, times, dict(zip(names, stages.tolist()))


def stages(x, fs, f0_floor=71.0, f0_ceil=800.0, *, device=0):
    """Intermediate stage buffers of one clip (diagnostic; see
    ``hv_harvest_stages``). Candidate arrays are expanded to the overlapped
    column layout of the reference's RefineF0Candidates input."""
    x = _check_array(x)
    fs = _as_int(fs, "fs")
    ratio = min(12, max(1, int(fs / 8000.0 + 0.5)))
    y_len = -(-x.size // ratio)
    frames = output_length(x.size, fs, 1.0)
    bands = 1 + int(np.log(f0_ceil * 1.1 / (f0_floor * 0.9)) / 0.69314718055994529 * 40.0)
    group = int(bands / 10.0 + 0.5)
    cap = 7 * group
    out = dict(y=np.zeros(y_len), raw=np.zeros((bands, frames)), cand_raw=np.zeros((frames, group)),
               refined=np.zeros((frames, cap)), scores=np.zeros((frames, cap)),
               pruned=np.zeros((frames, cap)), pruned_scores=np.zeros((frames, cap)),
               best=np.zeros(frames), smoothed=np.zeros(frames))
    count = np.zeros(1, dtype=np.int32)
    p = {k: v.ctypes.data_as(_D) for k, v in out.items()}
    status = _native.lib.hv_harvest_stages(
        x.ctypes.data_as(_D), x.size, fs, float(f0_floor), float(f0_ceil), _as_int(device, "device"),
        p["y"], p["raw"], count.ctypes.data_as(ct.POINTER(ct.c_int)), p["cand_raw"], p["refined"],
        p["scores"], p["pruned"], p["pruned_scores"], p["best"], p["smoothed"])
    _native.raise_for(status)
    k = int(count[0])
    cand = np.zeros((frames, cap))
    for g in range(7):
        shift = 0 if g == 0 else (g if g <= 3 else -(g - 3))
        for j in range(k):
            col = g * k + j
            src = np.arange(frames) - shift
            ok = (src >= 0) & (src < frames)
            cand[ok, col] = out["cand_raw"][src[ok], j]
    out["cand"] = cand
    out["count"] = k
    return out


def contour_batch(f0_candidates, scores, frame_offsets, columns=None, base=None, *, device=0):
    """FixF0Contour and SmoothF0Contour of the engine's contour stage on
    caller-given candidates (see ``hv_contour_batch``). ``f0_candidates``
    and ``scores`` are float64 ``[frames, stride]`` arrays holding every
    clip's rows back to back, ``frame_offsets`` (clips + 1 entries, from 0)
    delimits the clips, and the first ``columns`` columns (default: all) are
    the candidates. ``base`` (float64 ``[frames]``) replaces SearchF0Base's
    contour as the input of FixStep1. Returns ``(fixed, smoothed)``."""
    cand = np.ascontiguousarray(f0_candidates, dtype=np.float64)
    sc = np.ascontiguousarray(scores, dtype=np.float64)
    if cand.ndim != 2 or sc.shape != cand.shape:
        raise ValueError("f0_candidates and scores must be 2-D arrays of the same shape")
    frames, stride = cand.shape
    if stride == 0:        # no candidate columns: one zero column keeps the rows addressable
        cand, sc, stride, columns = np.zeros((frames, 1)), np.zeros((frames, 1)), 1, 0
    columns = stride if columns is None else _as_int(columns, "columns")
    off = np.ascontiguousarray(frame_offsets, dtype=np.int64)
    if off.ndim != 1 or off.size < 2 or off[0] != 0 or off[-1] != frames:
        raise ValueError("frame_offsets must run from 0 to the number of rows")
    b = None
    if base is not None:
        b = np.ascontiguousarray(base, dtype=np.float64)
        if b.shape != (frames,):
            raise ValueError("base must hold one value per row")
    fixed, smoothed = np.zeros(frames), np.zeros(frames)
    status = _native.lib.hv_contour_batch(
        cand.ctypes.data, sc.ctypes.data, None if b is None else b.ctypes.data,
        off.ctypes.data_as(ct.POINTER(ct.c_int64)), off.size - 1, columns, stride,
        _as_int(device, "device"), fixed.ctypes.data, smoothed.ctypes.data, 0, None)
    _native.raise_for(status)
    return fixed, smoothed


def _out_offsets(offsets, fs, frame_period):
    lens = [output_length(int(offsets[i + 1] - offsets[i]), fs, frame_period)
            for i in range(len(offsets) - 1)]
    out = np.zeros(len(lens) + 1, dtype=np.int64)
    out[1:] = np.cumsum(lens)
    return out


def harvest_batch(x, offsets, fs, f0_floor=71.0, f0_ceil=800.0, frame_period=5.0, *, device=0,
                  graph=True):
    """Harvest on many clips at once.

    ``x`` is one contiguous float64 array holding every clip back to back and
    ``offsets`` (int64, clips + 1) delimits them. Returns
    ``(f0, times, out_offsets)``: packed outputs and their offsets. The whole
    batch runs as one launch sequence (a replayed CUDA graph when ``graph``).
    """
    x = _check_array(x)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    if offsets.ndim != 1 or offsets.size < 2:
        raise ValueError("offsets must hold clips + 1 entries")
    if offsets[0] < 0 or offsets[-1] > x.size or np.any(np.diff(offsets) < 0):
        raise ValueError("offsets must be nondecreasing and lie within x")
    fs = _as_int(fs, "fs")
    device = _as_int(device, "device")
    frame_period = _as_float(frame_period, "frame_period")
    for i in range(offsets.size - 1):
        n = int(offsets[i + 1] - offsets[i])
        if n <= 0:
            raise ValueError(f"clip {i} is empty")
    out_off = _out_offsets(offsets, fs, frame_period)
    f0 = np.empty(int(out_off[-1]))
    times = np.empty(int(out_off[-1]))
    flags = 0 if graph else _native.HV_NO_GRAPH
    status = _native.lib.hv_harvest_batch(
        x.ctypes.data, offsets.ctypes.data_as(ct.POINTER(ct.c_int64)), offsets.size - 1, fs,
        _as_float(f0_floor, "f0_floor"), _as_float(f0_ceil, "f0_ceil"), frame_period, device,
        f0.ctypes.data, times.ctypes.data, flags, None)
    _native.raise_for(status)
    return f0, times, out_off


def harvest_batch_pcm16(x, offsets, fs, f0_floor=71.0, f0_ceil=800.0, frame_period=5.0, *, device=0,
                        graph=True):
    """``harvest_batch`` on 16-bit PCM samples (a contiguous int16 array,
    e.g. the frames of a mono PCM16 WAV file). Each sample is taken as
    sample / 32768, on the device, so the result equals ``harvest_batch`` on
    ``x / 32768.0`` bit for bit while a quarter of the bytes cross PCIe."""
    if not isinstance(x, np.ndarray) or x.dtype != np.int16 or x.ndim != 1 or not x.flags.c_contiguous:
        raise TypeError("x must be a 1-D C-contiguous numpy.ndarray of int16")
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    if offsets.ndim != 1 or offsets.size < 2:
        raise ValueError("offsets must hold clips + 1 entries")
    if offsets[0] < 0 or offsets[-1] > x.size or np.any(np.diff(offsets) < 0):
        raise ValueError("offsets must be nondecreasing and lie within x")
    fs = _as_int(fs, "fs")
    device = _as_int(device, "device")
    frame_period = _as_float(frame_period, "frame_period")
    out_off = _out_offsets(offsets, fs, frame_period)
    f0 = np.empty(int(out_off[-1]))
    times = np.empty(int(out_off[-1]))
    flags = 0 if graph else _native.HV_NO_GRAPH
    status = _native.lib.hv_harvest_batch_pcm16(
        x.ctypes.data, offsets.ctypes.data_as(ct.POINTER(ct.c_int64)), offsets.size - 1, fs,
        _as_float(f0_floor, "f0_floor"), _as_float(f0_ceil, "f0_ceil"), frame_period, device,
        f0.ctypes.data, times.ctypes.data, flags, None)
    _native.raise_for(status)
    return f0, times, out_off


def harvest_many(clips, fs, f0_floor=71.0, f0_ceil=800.0, frame_period=5.0, *, device=0,
                 graph=True):
    """``harvest`` on a list of clips in one batch; returns a list of
    ``(f0, times)`` pairs in clip order."""
    clips = [_check_array(c) for c in clips]
    offsets = np.zeros(len(clips) + 1, dtype=np.int64)
    offsets[1:] = np.cumsum([c.size for c in clips])
    packed = np.concatenate(clips) if clips else np.zeros(0)
    f0, times, out = harvest_batch(packed, offsets, fs, f0_floor, f0_ceil, frame_period,
                                   device=device, graph=graph)
    return [(f0[out[i]:out[i + 1]].copy(), times[out[i]:out[i + 1]].copy())
            for i in range(len(clips))]
