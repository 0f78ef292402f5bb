"""Accuracy metrics between two F0 tracks, as the reference's benchmark
reports them (reference benchmarks/benchmark.py:20-37): voicing
disagreement and pitch error in cents over jointly voiced frames."""
from __future__ import annotations

import numpy as np


def compare(reference, actual):
    reference = np.asarray(reference, dtype=np.float64)
    actual = np.asarray(actual, dtype=np.float64)
    if reference.shape != actual.shape:
        raise ValueError(f"Shape mismatch: {reference.shape} versus {actual.shape}")
    for name, f0 in (("reference", reference), ("actual", actual)):
        if not np.all(np.isfinite(f0)) or np.any(f0 < 0):
            raise ValueError(f"{name} F0 must contain only finite, nonnegative values")
    rv, av = reference > 0, actual > 0
    both = rv & av
    cents = np.abs(1200 * np.log2(actual[both] / reference[both]))
    rel = np.abs(actual[both] - reference[both]) / reference[both]
    return {
        "frames": int(reference.size),
        "reference_voiced_frames": int(rv.sum()),
        "joint_voiced_frames": int(both.sum()),
        "vuv_disagreement": float(np.mean(rv != av)) if reference.size else 0.0,
        "cents_p99": float(np.quantile(cents, 0.99)) if cents.size else None,
        "cents_max": float(cents.max()) if cents.size else None,
        "over_600_cents": int((cents > 600).sum()),
        "rel_max": float(rel.max()) if rel.size else None,
        "rel_frac_over_1e-6": float(np.mean(rel > 1e-6)) if rel.size else 0.0,
    }


_STAT_KEYS = ("frames", "reference_voiced_frames", "joint_voiced_frames", "vuv_disagreement",
              "cents_p99", "cents_max", "over_600_cents")


def compare_batch(reference, actual, offsets, *, device=0):
    """``compare`` for every clip of a packed batch, computed on the GPU
    (``hv_compare_batch``); clip c spans ``[offsets[c], offsets[c+1])``.

    NumPy inputs return a list of dicts with the keys of the reference's
    benchmark comparison (``cents_p99``/``cents_max`` are None for clips
    without jointly voiced frames). CUDA tensors are compared in place on
    their device and the call returns a ``(clips, 7)`` float64 CUDA tensor in
    the key order above, without waiting for the GPU."""
    import ctypes as ct

    from . import _native
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    clips = offsets.size - 1
    if clips < 1:
        raise ValueError("offsets must hold clips + 1 entries")
    off_ptr = offsets.ctypes.data_as(ct.POINTER(ct.c_int64))
    if hasattr(reference, "is_cuda") and reference.is_cuda:
        import torch
        if not (actual.is_cuda and reference.dtype == actual.dtype == torch.float64):
            raise TypeError("both tracks must be float64 CUDA tensors")
        reference, actual = reference.contiguous(), actual.contiguous()
        if offsets[-1] > min(reference.numel(), actual.numel()):
            raise ValueError("offsets exceed the tracks")
        stats = torch.empty((clips, 7), dtype=torch.float64, device=reference.device)
        stream = torch.cuda.current_stream(reference.device).cuda_stream
        _native.raise_for(_native.lib.hv_compare_batch(
            reference.data_ptr(), actual.data_ptr(), off_ptr, clips, reference.device.index, stats.data_ptr(),
            _native.HV_DEVICE_POINTERS | _native.HV_NULL_IS_LEGACY_STREAM, ct.c_void_p(stream or None)))
        return stats
    reference = np.ascontiguousarray(reference, dtype=np.float64)
    actual = np.ascontiguousarray(actual, dtype=np.float64)
    if reference.shape != actual.shape or offsets[-1] > reference.size:
        raise ValueError("the tracks must have equal shapes covering the offsets")
    stats = np.empty((clips, 7))
    _native.raise_for(_native.lib.hv_compare_batch(
        reference.ctypes.data, actual.ctypes.data, off_ptr, clips, int(device), stats.ctypes.data, 0, None))
    out = []
    for row in stats:
        d = dict(zip(_STAT_KEYS, row.tolist()))
        for k in ("frames", "reference_voiced_frames", "joint_voiced_frames", "over_600_cents"):
            d[k] = int(d[k])
        for k in ("cents_p99", "cents_max"):
            if np.isnan(d[k]):
                d[k] = None
        out.append(d)
    return out
