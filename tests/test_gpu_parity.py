"""Parity of the CUDA engine with the CPU checker (the reference's bundled
WORLD build when present). Ports the reference's GPU tests
(tests/test_compatibility.py) with pyworld replaced by that checker.

Acceptance: time axis bit-exact, voiced/unvoiced agreement >= 99.9 % of
frames and voiced F0 within 1e-6 relative; where the reference's own tests
use assert_allclose(rtol=1e-7, atol=1e-5) the same bound is kept."""
import json
import os

import numpy as np
import pytest

import harvest_cuda_b200 as hv
from harvest_cuda_b200 import signals
from harvest_cuda_b200.metrics import compare

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
F0_RTOL = 1e-6      # voiced F0, relative
VUV_MAX = 0.001     # fraction of frames whose voicing may differ


def assert_parity(actual, expected):
    (f0, t), (rf0, rt) = actual, expected
    np.testing.assert_array_equal(t, rt)
    m = compare(rf0, f0)
    assert m["vuv_disagreement"] <= VUV_MAX, m
    if m["joint_voiced_frames"]:
        both = (f0 > 0) & (rf0 > 0)
        rel = np.abs(f0[both] - rf0[both]) / rf0[both]
        # Frames whose voicing decision flipped are covered by VUV_MAX; every
        # jointly voiced frame must meet the F0 bound, with no allowance.
        assert rel.max() <= F0_RTOL, (float(rel.max()), int(np.argmax(rel)), m)
    return m


@pytest.mark.parametrize("fs", [8000, 16000, 24000, 44100, 48000])
@pytest.mark.parametrize("kind", ["speechlike", "low", "high", "noise", "silence"])
def test_matches_checker(gpu, checker, fs, kind):
    x = signals.kind_clip(kind, 0.7, fs)
    actual = hv.harvest(x, fs)
    assert actual[0].dtype == np.float64
    m = assert_parity(actual, checker.harvest(x, fs))
    if kind in ("low", "high", "speechlike"):
        assert m["joint_voiced_frames"] > 0


def test_golden_fixtures(gpu):
    with open(os.path.join(GOLDEN, "index.json")) as f:
        index = json.load(f)
    for case in index["cases"]:
        data = np.load(os.path.join(GOLDEN, case["file"]))
        actual = hv.harvest(data["x"], case["fs"], case["f0_floor"], case["f0_ceil"],
                            case["frame_period"])
        assert_parity(actual, (data["f0"], data["times"]))


@pytest.mark.parametrize("period,floor,ceil", [(1.0, 50, 900), (2.5, 100, 400), (7.3, 65, 1000)])
def test_parameters_and_readonly_input(gpu, checker, period, floor, ceil):
    x = signals.kind_clip("speechlike", 1.1, 44100)
    x.flags.writeable = False
    expected = checker.harvest(x, 44100, floor, ceil, period)
    actual = hv.harvest(x, 44100, floor, ceil, period)
    np.testing.assert_array_equal(actual[1], expected[1])
    np.testing.assert_allclose(actual[0], expected[0], rtol=1e-7, atol=1e-5)


@pytest.mark.parametrize("length", [6, 24, 240])
def test_short_silent_input(gpu, checker, length):
    x = np.zeros(length)
    expected = checker.harvest(x, 24000)
    actual = hv.harvest(x, 24000)
    np.testing.assert_array_equal(actual[0], expected[0])
    np.testing.assert_array_equal(actual[1], expected[1])


@pytest.mark.parametrize("seconds,fs,period", [(4.0, 16000, 5.0), (9.0, 44100, 1.0)])
def test_long_voiced_section(gpu, checker, seconds, fs, period):
    # One voiced section longer than 2048 frames: the engine smooths it with
    # the whole warp in warmed-up chunks instead of one sequential pass; its
    # F0 must stay within rounding of the sequential result.
    x = signals.glide_clip(seconds, fs, edge=0.2, seed=12)[0]
    expected = checker.harvest(x, fs, 71.0, 800.0, period)
    actual = hv.harvest(x, fs, 71.0, 800.0, period)
    assert np.count_nonzero(expected[0]) * period > 2100
    np.testing.assert_array_equal(actual[1], expected[1])
    both = (actual[0] > 0) & (expected[0] > 0)
    assert np.array_equal(actual[0] > 0, expected[0] > 0)
    assert np.max(np.abs(actual[0][both] - expected[0][both]) / expected[0][both]) <= 1e-10


def _limit_cycle_period(x):
    """Period of the state orbit of the smoothing filter (FilteringF0's
    recursive part) on the constant input x from a zero state: 1 for a fixed
    point, more for a rounding limit cycle."""
    a0, a1 = 1.7347257688092754, -0.76600660094326412
    w0 = w1 = 0.0
    seen = {}
    for k in range(3000):
        if (w0, w1) in seen:
            return k - seen[(w0, w1)]
        seen[(w0, w1)] = k
        w0, w1 = x + a0 * w0 + a1 * w1, w0
    return 0


def test_smoothing_of_held_limit_cycles(gpu, checker):
    # Twenty voiced sections at different pitches. Each section is smoothed
    # over the whole padded length with its first and last values held; on
    # such a constant input the filter state ends in a fixed point or, for
    # about a fifth of the values, in a rounding limit cycle, whose whole
    # periods the engine skips. Its smoothed contour must equal the oracle's
    # smoothing of the engine's own fixed contour bit for bit (all sections
    # are shorter than 2048 frames).
    fs, sections = 16000, 20
    t = np.arange(int(fs * 0.3 * sections)) / fs
    x = np.zeros_like(t)
    for s in range(sections):
        on = (t >= 0.3 * s) & (t < 0.3 * s + 0.18)
        x[on] = sum(np.sin(2 * np.pi * (90.0 + 17.0 * s) * h * t[on]) / h for h in range(1, 6))
    g = hv.api.stages(x, fs)
    fixed = checker.fix_contour(g["pruned"], g["pruned_scores"], 7 * g["count"])
    np.testing.assert_array_equal(g["smoothed"], checker.smooth_contour(fixed))
    d = np.diff(np.concatenate([[0], (fixed > 0).astype(int), [0]]))
    heads = fixed[np.flatnonzero(d == 1)]
    assert len(heads) >= 15
    assert sum(_limit_cycle_period(float(v)) > 1 for v in heads) >= 2


def test_separate_voiced_sections(gpu, checker):
    fs = 16000
    t = np.arange(fs * 8) / fs
    x = sum(np.sin(2 * np.pi * 137 * h * t) / h for h in range(1, 6))
    x[(t % 0.8 > 0.5) & (t < 7.5)] = 0
    expected = checker.harvest(x, fs)
    actual = hv.harvest(x, fs)
    assert np.count_nonzero(expected[0]) > 100
    assert np.count_nonzero(expected[0] == 0) > 100
    np.testing.assert_array_equal(actual[1], expected[1])
    np.testing.assert_allclose(actual[0], expected[0], rtol=1e-7, atol=1e-5)


@pytest.mark.parametrize("fs,frequency,floor,ceil", [
    (8000, 16, 8, 90),        # long refinement windows (FFT size 8192 in WORLD)
    (11025, 30, 10, 100),
    (192000, 75, 40, 250),    # internal rate above 8 kHz
    (8000, 2400, 1200, 3900),  # fewer than six harmonics
])
def test_refinement_window_sizes(gpu, checker, fs, frequency, floor, ceil):
    seconds = 4.3 if frequency < 40 else 1.6
    t = np.arange(round(seconds * fs)) / fs
    pitch = frequency * (1 + 0.2 * np.sin(2 * np.pi * 0.7 * t))
    phase = 2 * np.pi * np.cumsum(pitch) / fs
    harmonics = min(6, int(fs / (2 * frequency * 1.2)))
    x = sum(0.2 * np.sin(h * phase + 0.1 * h) / h for h in range(1, harmonics + 1))
    x += np.random.default_rng(456).normal(0, 0.0001, len(t))
    expected = checker.harvest(x, fs, floor, ceil)
    for _ in range(2):
        actual = hv.harvest(x, fs, floor, ceil)
        np.testing.assert_array_equal(actual[1], expected[1])
        np.testing.assert_allclose(actual[0], expected[0], rtol=1e-7, atol=1e-5)


@pytest.mark.parametrize("fs", [16000, 24000, 32000, 40000, 48000, 56000, 64000, 72000, 80000,
                                88000, 96000, 192000, 44100])
def test_every_decimation_ratio(gpu, checker, fs):
    x = signals.kind_clip("speechlike", 2.1, fs)[:-1]
    expected = checker.harvest(x, fs)
    actual = hv.harvest(x, fs)
    np.testing.assert_array_equal(actual[1], expected[1])
    np.testing.assert_allclose(actual[0], expected[0], rtol=1e-7, atol=1e-5)


@pytest.mark.parametrize("fs", [72000, 80000, 192000])
@pytest.mark.parametrize("constant", [True, False])
def test_dc_input(gpu, checker, fs, constant):
    # Valid output without reproducing WORLD's rounding artifacts on DC.
    x = np.ones(round(2.2 * fs)) if constant else 1000 + 0.01 * signals.kind_clip("speechlike", 2.2, fs)
    expected = checker.harvest(x, fs)
    actual = hv.harvest(x, fs)
    np.testing.assert_array_equal(actual[1], expected[1])
    assert np.all(np.isfinite(actual[0])) and np.all(actual[0] >= 0)


@pytest.mark.parametrize("length", [24576, 24577, 24578, 24800])
def test_final_bin_correction(gpu, checker, length):
    # Excites the two whole-signal spectrum bins WORLD overwrites.
    fs = 8000
    x = signals.kind_clip("speechlike", length / fs, fs)
    i = np.arange(x.size)
    x = x + 0.01 * ((1 - 2 * (i % 2)) + np.cos(2 * np.pi * (0.5 - 1 / 32768) * i))
    expected = checker.harvest(x, fs)
    actual = hv.harvest(x, fs)
    np.testing.assert_array_equal(actual[1], expected[1])
    np.testing.assert_allclose(actual[0], expected[0], rtol=1e-7, atol=1e-5)


def test_stage_parity(gpu, checker):
    # Stage by stage on one clip: candidate count equal, no voicing flips in
    # any candidate matrix, values within 1e-9 relative.
    x = signals.kind_clip("speechlike", 0.7, 16000)
    g = hv.api.stages(x, 16000)
    r = checker.stages(x, 16000)
    assert g["count"] == r["count"]
    np.testing.assert_allclose(g["y"], r["y"], rtol=0, atol=1e-12 * np.abs(r["y"]).max())
    for key, rkey in [("raw", "raw"), ("cand", "cand"), ("refined", "refined"), ("pruned", "pruned"),
                      ("best", "base"), ("smoothed", "smoothed")]:
        a, b = g[key], r[rkey]
        assert np.array_equal(a != 0, b != 0), key
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=0, err_msg=key)


def test_deterministic(gpu):
    x = signals.kind_clip("speechlike", 1.3, 22050)
    first = hv.harvest(x, 22050)
    for _ in range(2):
        again = hv.harvest(x, 22050)
        np.testing.assert_array_equal(again[0], first[0])
        np.testing.assert_array_equal(again[1], first[1])


def test_direct_fir_bank_matches_fft_bank(gpu, checker, monkeypatch):
    # The engine picks the overlap-save FFT bank unless the filters are too
    # long for it; force the direct FIR bank and compare both with the checker.
    x = signals.kind_clip("speechlike", 1.3, 16000)
    fft = hv.harvest(x, 16000)
    monkeypatch.setenv("HARVEST_B200_BANK", "fir")
    hv.clear_cache()
    fir = hv.harvest(x, 16000)
    monkeypatch.delenv("HARVEST_B200_BANK")
    hv.clear_cache()
    expected = checker.harvest(x, 16000)
    for actual in (fft, fir):
        np.testing.assert_array_equal(actual[1], expected[1])
        np.testing.assert_allclose(actual[0], expected[0], rtol=1e-7, atol=1e-5)
