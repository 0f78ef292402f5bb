"""On-device accuracy metrics (hv_compare_batch) against the NumPy
comparison of the reference's benchmark, clip by clip."""
import numpy as np
import pytest

from harvest_cuda_b200.metrics import compare, compare_batch

pytestmark = pytest.mark.gpu


def _tracks(rng, n):
    ref = np.where(rng.random(n) < 0.7, rng.uniform(60, 600, n), 0.0)
    act = np.where(rng.random(n) < 0.95, ref * np.exp2(rng.normal(0, 0.01, n)), 0.0)
    act[rng.random(n) < 0.02] = rng.uniform(60, 600)          # some gross errors
    act[(ref == 0) & (rng.random(n) < 0.05)] = 200.0          # some false voicing
    return ref, act


def test_matches_numpy_comparison_per_clip(gpu):
    rng = np.random.default_rng(2)
    lengths = [0, 1, 5, 301, 4097, 30001, 12]
    parts = [_tracks(rng, n) for n in lengths]
    parts.append((np.zeros(50), np.full(50, 120.0)))          # no jointly voiced frame
    ref = np.concatenate([p[0] for p in parts])
    act = np.concatenate([p[1] for p in parts])
    offsets = np.concatenate([[0], np.cumsum([len(p[0]) for p in parts])])
    got = compare_batch(ref, act, offsets)
    for (r, a), g in zip(parts, got):
        if r.size == 0:
            assert g["frames"] == 0 and g["joint_voiced_frames"] == 0
            continue
        want = compare(r, a)
        for k in ("frames", "reference_voiced_frames", "joint_voiced_frames", "over_600_cents"):
            assert g[k] == want[k], k
        assert g["vuv_disagreement"] == pytest.approx(want["vuv_disagreement"], rel=1e-15)
        for k in ("cents_p99", "cents_max"):
            if want[k] is None:
                assert g[k] is None
            else:
                assert g[k] == pytest.approx(want[k], rel=1e-12, abs=1e-12), k


def test_device_tensors(gpu):
    import torch
    rng = np.random.default_rng(3)
    ref, act = _tracks(rng, 9000)
    offsets = [0, 3000, 9000]
    host = compare_batch(ref, act, offsets)
    dev = compare_batch(torch.from_numpy(ref).cuda(), torch.from_numpy(act).cuda(), offsets).cpu().numpy()
    for row, h in zip(dev, host):
        assert row[0] == h["frames"] and row[2] == h["joint_voiced_frames"] and row[6] == h["over_600_cents"]
        assert row[4] == h["cents_p99"] and row[5] == h["cents_max"]
