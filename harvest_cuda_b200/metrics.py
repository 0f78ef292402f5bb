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
