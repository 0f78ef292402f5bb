"""The integer-key warp reductions of the contour kernels (`warp_pick`,
`warp_max_score` in harvest_cuda_b200/csrc/contour.cu), restated with NumPy
on the CPU and checked against the sequential loops they stand for:

* SelectBestF0 (reference third_party/world/src/harvest.cpp:636-650): the
  column of smallest |ref - c| / ref within `allowed`, the later column on
  ties, 0 if none; the warp version lets lane l scan columns l, l + 32, ...
  and then reduces the lanes' picks by order-preserving 64-bit keys (min of
  the high words, min of the low words among those, max column among
  those);
* the SearchScore maximum (harvest.cpp:901-907): a lane keeps a score only
  when it exceeds its current maximum (starting at 0), so the partial maxima
  are +0 or larger and never NaN, and the lanes' maximum is taken on the
  high and then the low word of their bit patterns.
"""
import numpy as np

LANES = 32


def _key(e):
    """Unsigned key of a double in the same order (-0 as +0), as warp_pick
    forms it."""
    b = np.array([e + 0.0], dtype=np.float64).view(np.uint64)[0]
    return np.uint64(~b) if b >> np.uint64(63) else np.uint64(b | np.uint64(1 << 63))


def _select_best_sequential(ref, row, allowed):
    best_e, pick = allowed, 0.0
    for c in row:
        e = abs(ref - c) / ref
        if e <= best_e:
            best_e, pick = e, c
    return pick


def _select_best_warp(ref, row, allowed):
    picks = []
    for lane in range(LANES):
        best_e, best_i, val = allowed, -1, 0.0
        for i in range(lane, len(row), LANES):
            e = abs(ref - row[i]) / ref
            if e <= best_e:
                best_e, best_i, val = e, i, row[i]
        key = _key(best_e) if best_i >= 0 else np.uint64(2**64 - 1)
        picks.append((int(key >> np.uint64(32)), int(key & np.uint64(0xFFFFFFFF)), best_i, val))
    min_hi = min(p[0] for p in picks)
    min_lo = min(p[1] if p[0] == min_hi else 0xFFFFFFFF for p in picks)
    top = max((p[2] + 1) if (p[2] >= 0 and p[0] == min_hi and p[1] == min_lo) else 0 for p in picks)
    return picks[(top - 1) % LANES][3] if top else 0.0


def _max_score_warp(value, row, scores):
    parts = []
    for lane in range(LANES):
        s = 0.0
        for i in range(lane, len(row), LANES):
            if value == row[i] and s < scores[i]:
                s = scores[i]
        parts.append(np.array([s], dtype=np.float64).view(np.uint64)[0])
    his = [int(b >> np.uint64(32)) for b in parts]
    los = [int(b & np.uint64(0xFFFFFFFF)) for b in parts]
    max_hi = max(his)
    max_lo = max(lo if hi == max_hi else 0 for hi, lo in zip(his, los))
    return np.array([(max_hi << 32) | max_lo], dtype=np.uint64).view(np.float64)[0]


def _max_score_sequential(value, row, scores):
    s = 0.0
    for c, sc in zip(row, scores):
        if value == c and s < sc:
            s = sc
    return s


def test_key_order_matches_double_order():
    rng = np.random.default_rng(5)
    vals = np.concatenate([rng.standard_normal(300) * 10.0 ** rng.integers(-300, 300, 300),
                           [0.0, -0.0, np.inf, -np.inf, 5e-324, -5e-324, 0.18, -0.18]])
    keys = [_key(v) for v in vals]
    for a in range(len(vals)):
        for b in range(0, len(vals), 7):
            assert (vals[a] < vals[b]) == (keys[a] < keys[b])
            assert (vals[a] == vals[b]) == (keys[a] == keys[b])


def test_warp_pick_matches_select_best():
    rng = np.random.default_rng(11)
    for trial in range(400):
        n = int(rng.integers(1, 300))
        ref = float(rng.uniform(60, 900)) * (-1.0 if trial % 17 == 0 else 1.0)
        base = rng.uniform(50, 1000, size=n)
        # Ties: repeated values and values equally far above and below ref.
        if trial % 3 == 0:
            base[rng.integers(0, n, size=n // 3 + 1)] = ref * (1 + rng.choice([-0.05, 0.05, 0.0, 0.18]))
        if trial % 5 == 0:
            base[rng.integers(0, n, size=n // 4 + 1)] = 0.0
        allowed = [0.18, 0.008, 0.05][trial % 3]
        row = list(base)
        assert _select_best_warp(ref, row, allowed) == _select_best_sequential(ref, row, allowed)


def test_warp_max_score_matches_the_running_maximum():
    rng = np.random.default_rng(13)
    for trial in range(300):
        n = int(rng.integers(1, 300))
        row = rng.choice([110.0, 220.0, 330.0, 0.0], size=n)
        scores = rng.uniform(0, 50, size=n)
        if trial % 4 == 0:
            scores[rng.integers(0, n, size=n // 5 + 1)] = np.nan
        if trial % 6 == 0:
            scores[rng.integers(0, n, size=2)] = np.inf
        if trial % 7 == 0:
            scores[rng.integers(0, n, size=3)] = -0.0
        value = float(rng.choice([110.0, 220.0, 330.0, 440.0]))
        want = _max_score_sequential(value, row, scores)
        got = _max_score_warp(value, row, scores)
        assert np.array([got]).view(np.uint64)[0] == np.array([want]).view(np.uint64)[0]
