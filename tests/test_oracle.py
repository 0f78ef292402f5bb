"""Pins the C restatement of Harvest (oracle/harvest_oracle.c) against the
reference's own bundled WORLD build (oracle/_ref) and against the committed
golden fixtures. CPU only."""
import json
import os

import numpy as np
import pytest

import oracle
from harvest_cuda_b200 import signals
from harvest_cuda_b200.metrics import compare

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _ref():
    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference build oracle/_ref absent")
    return ref


@pytest.mark.parametrize("fs", [8000, 16000, 24000, 44100, 48000])
@pytest.mark.parametrize("period", [1.0, 2.5, 5.0, 10.0])
def test_port_matches_reference_world(fs, period):
    # The reference's own oracle test shape (tests/test_compatibility.py:9-22):
    # 0.35 s of a speech-like signal, times exact, f0 at rtol 1e-10.
    x = signals.kind_clip("speechlike", 0.35, fs)
    f0_ref, t_ref = _ref().harvest(x, fs, frame_period=period)
    f0, t = oracle.port().harvest(x, fs, frame_period=period)
    np.testing.assert_array_equal(t, t_ref)
    np.testing.assert_allclose(f0, f0_ref, rtol=1e-10, atol=1e-8)


@pytest.mark.parametrize("kind", ["low", "high", "noise", "silence"])
def test_port_matches_reference_world_kinds(kind):
    x = signals.kind_clip(kind, 0.5, 16000)
    f0_ref, t_ref = _ref().harvest(x, 16000)
    f0, t = oracle.port().harvest(x, 16000)
    np.testing.assert_array_equal(t, t_ref)
    np.testing.assert_allclose(f0, f0_ref, rtol=1e-10, atol=1e-8)


def test_port_decimation_is_bit_exact():
    for fs in (16000, 24000, 44100, 48000, 96000, 192000):
        x = signals.kind_clip("speechlike", 0.2, fs)
        assert np.array_equal(oracle.port().stages(x, fs)["y"], _ref().stages(x, fs)["y"])


def test_port_stage_parameters_match():
    for n, fs, lo, hi in [(48000, 16000, 71, 800), (2646000, 44100, 71, 800),
                          (16000, 16000, 50, 1100), (1440000, 48000, 71, 800), (6, 24000, 71, 800)]:
        assert oracle.port().params(n, fs, lo, hi) == _ref().params(n, fs, lo, hi)


def _random_tracks(rng, frames, columns):
    pitches = np.array([80, 90, 120, 150, 180, 250, 400, 600], dtype=float)
    f0 = np.zeros((frames, columns))
    scores = np.zeros((frames, columns))
    for col in range(columns):
        period, gap, phase = rng.integers(10, 160), rng.integers(0, 8), rng.integers(0, 160)
        voiced = (np.arange(frames) + phase) % period >= gap
        f0[voiced, col] = pitches[col % 8] * (1 + 0.01 * rng.standard_normal(voiced.sum()))
        scores[voiced, col] = rng.integers(1, 11, voiced.sum())
    return f0, scores


def test_port_contour_matches_reference_exactly():
    # FixF0Contour on synthetic candidate tracks must agree bit for bit, the
    # check the reference's own tests/cpp/test_contour.cpp:116-151 makes.
    rng = np.random.default_rng(20261110)
    for trial in range(200):
        frames = int(rng.integers(2, 1500))
        f0, scores = _random_tracks(rng, frames, 8)
        if trial % 10 == 0:
            f0[:] = 0
            scores[:] = 0
        a = oracle.port().fix_contour(f0, scores)
        b = _ref().fix_contour(f0, scores)
        assert np.array_equal(a, b), trial
        assert np.array_equal(oracle.port().smooth_contour(a), _ref().smooth_contour(b)), trial


def test_golden_fixtures():
    # Fixtures made by tests/golden/make_golden.py from the reference build.
    with open(os.path.join(GOLDEN, "index.json")) as f:
        index = json.load(f)
    for case in index["cases"]:
        data = np.load(os.path.join(GOLDEN, case["file"]))
        x = data["x"]
        f0, t = oracle.port().harvest(x, case["fs"], case["f0_floor"], case["f0_ceil"],
                                      case["frame_period"])
        np.testing.assert_array_equal(t, data["times"])
        m = compare(data["f0"], f0)
        assert m["vuv_disagreement"] == 0.0, case["file"]
        if m["joint_voiced_frames"]:
            assert m["rel_max"] < 1e-9, case["file"]
