"""The engine's contour kernel (FixF0Contour + SmoothF0Contour, one warp per
clip) on adversarial candidate matrices, bit for bit against the CPU checker
(the reference's bundled WORLD build when present), through
``hv_contour_batch``. The cases follow the reference's own contour checks
(tests/cpp/test_contour.cpp:64-151), generated here with NumPy:

* 1000 random trials of 2-2001 frames x 8 candidate tracks (seed 20261110):
  periodic voiced tracks with gaps that extension can and cannot cross,
  tracks at 8 or 4 distinct pitches, scores 1-10, and random voiced
  sections as the base contour (every tenth trial none); run both from
  SearchF0Base's contour and from the given base;
* SearchF0Base and SearchScore (MergeF0Sub's score sums) with NaN and
  infinite scores;
* ExtendF0 on candidates one ulp apart at 0.82, 1.18 and 1.001 times the
  section's value: the 18 % cutoff and ties between equally close
  candidates (WORLD keeps the later one), in both directions;
* no candidate columns at all, for 1, 2 and 1000 frames.

Every trial of a kind runs in one batched call (one warp per trial)."""
import numpy as np
import pytest

import harvest_cuda_b200 as hv
from harvest_cuda_b200.api import contour_batch

pytestmark = pytest.mark.gpu

PITCHES = np.array([80.0, 90.0, 120.0, 150.0, 180.0, 250.0, 400.0, 600.0])


def random_trial(rng, trial):
    frames = 2 + int(rng.integers(2000))
    cand = np.zeros((frames, 8))
    scores = np.zeros((frames, 8))
    rows = np.arange(frames)
    for col in range(8):
        period = 10 + int(rng.integers(150))
        gap = int(rng.integers(8))
        phase = int(rng.integers(period))
        voiced = np.full(frames, trial % 4 == 0) | ((rows + phase) % period >= gap)
        pitch = PITCHES[col % 4] if trial % 3 == 0 else PITCHES[col]
        cand[:, col] = np.where(voiced, pitch, 0.0)
        scores[:, col] = np.where(voiced, 1 + rng.integers(10, size=frames), 0.0)
    base = np.zeros(frames)
    start = 1
    while start < frames - 1:
        end = min(frames - 2, start + 6 + int(rng.integers(80)))
        base[start:end + 1] = PITCHES[rng.integers(8)]
        start = end + 2 + int(rng.integers(100))
    if trial % 10 == 0:
        base[:] = 0.0
    return cand, scores, base


def run_batch(trials, use_base, columns=None):
    """All trials through one GPU call; returns per-trial (fixed, smoothed)."""
    lengths = [t[0].shape[0] for t in trials]
    off = np.concatenate([[0], np.cumsum(lengths)]).astype(np.int64)
    cand = np.concatenate([t[0] for t in trials])
    scores = np.concatenate([t[1] for t in trials])
    base = np.concatenate([t[2] for t in trials]) if use_base else None
    fixed, smoothed = contour_batch(cand, scores, off, columns=columns, base=base)
    return [(fixed[a:b], smoothed[a:b]) for a, b in zip(off[:-1], off[1:])]


def expect_equal(checker, trials, results, use_base, columns=None):
    for k, ((cand, scores, base), (fixed, smoothed)) in enumerate(zip(trials, results)):
        want = checker.fix_contour(cand, scores, columns=columns, base=base if use_base else None)
        np.testing.assert_array_equal(fixed, want, err_msg=f"FixF0Contour, trial {k}")
        np.testing.assert_array_equal(smoothed, checker.smooth_contour(want),
                                      err_msg=f"SmoothF0Contour, trial {k}")


@pytest.fixture(scope="module")
def random_trials():
    rng = np.random.default_rng(20261110)
    return [random_trial(rng, t) for t in range(1000)]


@pytest.mark.parametrize("use_base", [False, True], ids=["search_f0_base", "given_base"])
def test_random_trials(gpu, checker, random_trials, use_base):
    results = run_batch(random_trials, use_base)
    expect_equal(checker, random_trials, results, use_base)
    # SearchF0Base jumps between the tracks' pitches, so FixStep1 keeps
    # little of it; the given sections survive far more.
    voiced = sum(int(np.count_nonzero(f)) for f, _ in results)
    assert voiced > (100000 if use_base else 1000)


@pytest.mark.parametrize("use_base", [False, True], ids=["search_f0_base", "given_base"])
def test_nan_and_infinite_scores(gpu, checker, use_base):
    rng = np.random.default_rng(719)
    trials = []
    for t in range(200):
        cand, scores, base = random_trial(rng, t)
        voiced = scores > 0
        pick = rng.random(scores.shape)
        scores[voiced & (pick < 0.05)] = np.nan
        scores[voiced & (pick > 0.95)] = np.inf
        trials.append((cand, scores, base))
    results = run_batch(trials, use_base)
    expect_equal(checker, trials, results, use_base)


def ulp_trial(rng, trial):
    """A voiced section of one value with, at the frames next to its ends,
    eight candidates one ulp apart at 0.82, 1.18 or 1.001 times it."""
    frames = 160
    reference = 20.0 + rng.integers(4_000_000) / 1000.0
    factor = (0.82, 1.18, 1.001)[trial % 3]
    cand = np.zeros((frames, 8))
    scores = np.zeros((frames, 8))
    base = np.zeros(frames)
    base[40:120] = reference
    cand[40:120, 0] = reference
    scores[40:120, 0] = 1.0
    toward = 0.0 if trial % 2 else 10000.0
    for row in (38, 39, 40, 120, 121):
        v = reference * factor
        values = []
        for _ in range(8):
            values.append(v)
            v = np.nextafter(v, toward)
        cand[row] = rng.permutation(values)
        scores[row] = 1.0 + rng.integers(10, size=8)
    return cand, scores, base


@pytest.mark.parametrize("use_base", [False, True], ids=["search_f0_base", "given_base"])
def test_adjacent_ulp_candidates(gpu, checker, use_base):
    rng = np.random.default_rng(20261110)
    trials = [ulp_trial(rng, t) for t in range(2000)]
    results = run_batch(trials, use_base)
    expect_equal(checker, trials, results, use_base)
    assert sum(int(np.count_nonzero(f)) for f, _ in results) > 1000


def test_no_candidate_columns(gpu, checker):
    for frames in (1, 2, 1000):
        trials = [(np.zeros((frames, 0)), np.zeros((frames, 0)), np.zeros(frames))]
        (fixed, smoothed), = run_batch(trials, False)
        np.testing.assert_array_equal(fixed, np.zeros(frames))
        np.testing.assert_array_equal(smoothed, np.zeros(frames))
        np.testing.assert_array_equal(fixed, checker.fix_contour(*trials[0][:2]))


def test_contour_batch_matches_pipeline(gpu, checker):
    # The stage entry on a real clip's pruned candidates reproduces the
    # pipeline's own contour (the stage dump of the same clip).
    from harvest_cuda_b200 import signals
    x, _ = signals.glide_clip(3.0, 16000, seed=11)
    st = hv.api.stages(x, 16000)
    columns = 7 * st["count"]
    fixed, smoothed = contour_batch(st["pruned"], st["pruned_scores"],
                                    np.array([0, st["pruned"].shape[0]]), columns=columns)
    np.testing.assert_array_equal(smoothed, st["smoothed"])
    np.testing.assert_array_equal(fixed, checker.fix_contour(st["pruned"], st["pruned_scores"], columns=columns))


def test_contour_batch_rejects_bad_arguments(gpu):
    cand = np.zeros((10, 4))
    with pytest.raises(ValueError):
        contour_batch(cand, cand, np.array([0, 5]))            # offsets do not cover the rows
    with pytest.raises(ValueError):
        contour_batch(cand, cand, np.array([0, 10]), columns=5)   # more columns than the stride
    with pytest.raises(ValueError):
        contour_batch(cand, cand, np.array([0, 0, 10]))        # an empty clip


def test_extend_sub_decisions_on_the_threshold(gpu, checker):
    # ExtendSub keeps a section when 2200 / mean < its extended length n.
    # A section of value 2200 / n over exactly n summed frames sits on the
    # threshold, where the engine must fall back to the reference's ordered
    # sum; sections after it then carry that exact mean. With no candidates,
    # ExtendF0 stops at once: a base run over frames a..b becomes the
    # section a+1..b (FixStep1 drops its first frame), n = b - a - 1.
    trials = []
    for n, others in ((10, 0), (11, 2), (20, 3), (8, 1), (40, 4)):
        frames = 400
        base = np.zeros(frames)
        a = 20
        base[a:a + n + 2] = 2200.0 / n
        rng = np.random.default_rng(n)
        start = a + n + 12
        for _ in range(others):   # later sections, some on their own threshold
            m = int(rng.integers(8, 40))
            base[start:start + m + 2] = 2200.0 / m if rng.random() < 0.5 else float(rng.uniform(60, 600))
            start += m + 12
        trials.append((np.zeros((frames, 8)), np.zeros((frames, 8)), base))
    results = run_batch(trials, use_base=True)
    expect_equal(checker, trials, results, use_base=True)


def dense_trial(rng, trial):
    """Short given sections every few dozen frames, with every track holding
    one of two pitches at every frame, so that each section extends up to
    100 frames both ways and several extended sections overlap at once:
    MergeF0's decisions then depend on one another through long chains."""
    frames = 3000 + int(rng.integers(3000))
    pitches = (120.0, 150.0) if trial % 2 else (200.0, 203.0)
    cand = np.zeros((frames, 8))
    scores = np.zeros((frames, 8))
    for col in range(8):
        cand[:, col] = pitches[col % 2]
        scores[:, col] = 1 + rng.integers(10, size=frames)
    base = np.zeros(frames)
    start = 1 + int(rng.integers(20))
    while start < frames - 2:
        end = min(frames - 2, start + 7 + int(rng.integers(30)))
        base[start:end + 1] = pitches[int(rng.integers(2))]
        start = end + 2 + int(rng.integers(25))
    return cand, scores, base


@pytest.mark.parametrize("use_base", [False, True], ids=["search_f0_base", "given_base"])
def test_dense_overlapping_sections(gpu, checker, use_base):
    rng = np.random.default_rng(4242)
    trials = [dense_trial(rng, t) for t in range(60)]
    results = run_batch(trials, use_base)
    for k, ((cand, scores, base), (fixed, smoothed)) in enumerate(zip(trials, results)):
        want = checker.fix_contour(cand, scores, base=base if use_base else None)
        np.testing.assert_array_equal(fixed, want, err_msg=f"FixF0Contour, trial {k}")
        # Merged sections here reach 2048 frames and more, which the engine
        # smooths a warp at a time: equal to WORLD's pass up to rounding.
        np.testing.assert_allclose(smoothed, checker.smooth_contour(want), rtol=1e-12, atol=0,
                                   err_msg=f"SmoothF0Contour, trial {k}")
    assert sum(int(np.count_nonzero(f)) for f, _ in results) > 100000
