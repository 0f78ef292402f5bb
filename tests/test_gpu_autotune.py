"""The autotuner (the refinement's launch shape and the contour's section-
extension blocks per clip): every candidate gives bit-identical F0, tuning
runs once per (fs, f0 range, length buckets) and is then reused, and
HARVEST_B200_AUTOTUNE=0 falls back to the default shape."""
import ctypes as ct
import os

import numpy as np
import pytest

import harvest_cuda_b200 as hv
from harvest_cuda_b200 import _native, signals

pytestmark = pytest.mark.gpu

SHAPES = [(a, b) for a in (1, 4, 5) for b in (16, 32, 64)]


def _last_tuning():
    out = (ct.c_int * 3)()
    _native.raise_for(_native.lib.hv_last_tuning(out))
    return tuple(out)


@pytest.fixture
def clean_env():
    saved = {k: os.environ.get(k) for k in ("HARVEST_B200_AUTOTUNE", "HARVEST_B200_REFINE_SHAPE")}
    yield
    for k, v in saved.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v
    hv.clear_cache()


def _clips():
    return [signals.glide_clip(s, 16000, seed=i)[0] for i, s in enumerate((1.1, 2.3, 0.7, 3.2))]


def test_every_shape_gives_identical_f0(gpu, clean_env):
    clips = _clips()
    want = None
    for shape in SHAPES:
        hv.clear_cache()
        os.environ["HARVEST_B200_REFINE_SHAPE"] = f"{shape[0]},{shape[1]}"
        got = hv.harvest_many(clips, 16000, 50.0, 1100.0, 5.0)
        assert _last_tuning()[:2] == shape
        if want is None:
            want = got
        for (f0, t), (wf, wt) in zip(got, want):
            assert np.array_equal(f0, wf) and np.array_equal(t, wt), shape


def test_tuning_runs_once_per_key(gpu, clean_env):
    os.environ.pop("HARVEST_B200_REFINE_SHAPE", None)
    os.environ.pop("HARVEST_B200_AUTOTUNE", None)
    hv.clear_cache()
    clips = _clips()
    first = hv.harvest_many(clips, 16000, 50.0, 1100.0, 5.0)
    shape = _last_tuning()
    assert shape[2] == 1 and shape[:2] in SHAPES
    again = hv.harvest_many(clips, 16000, 50.0, 1100.0, 5.0)
    assert _last_tuning() == (shape[0], shape[1], 0)
    # Same key (length bucket) with other lengths: the plan is new, the shape is reused.
    hv.harvest_many([c[:-100] for c in clips], 16000, 50.0, 1100.0, 5.0)
    assert _last_tuning() == (shape[0], shape[1], 0)
    for (f0, t), (wf, wt) in zip(first, again):
        assert np.array_equal(f0, wf) and np.array_equal(t, wt)
    os.environ["HARVEST_B200_AUTOTUNE"] = "0"
    hv.clear_cache()
    off = hv.harvest_many(clips, 16000, 50.0, 1100.0, 5.0)
    assert _last_tuning() == (4, 32, 0)
    for (f0, t), (wf, wt) in zip(first, off):
        assert np.array_equal(f0, wf) and np.array_equal(t, wt)


def test_every_contour_block_count_gives_identical_f0(gpu, clean_env):
    # Noisy 48 kHz clips with 1 ms frames have hundreds of voiced sections,
    # which the contour's extension kernel spreads over its blocks.
    saved = os.environ.get("HARVEST_B200_CONTOUR_BLOCKS")
    try:
        clips, _ = signals.ragged_batch(6, 48000, (2.0, 5.0), f0_range=(60.0, 600.0), snr_range=(0.0, 3.0),
                                        seed=5)
        want = None
        for blocks in (1, 3, 8, 32):
            hv.clear_cache()
            os.environ["HARVEST_B200_CONTOUR_BLOCKS"] = str(blocks)
            got = hv.harvest_many(clips, 48000, 71.0, 800.0, 1.0)
            if want is None:
                want = got
            for (f0, t), (wf, wt) in zip(got, want):
                assert np.array_equal(f0, wf) and np.array_equal(t, wt), blocks
    finally:
        if saved is None:
            os.environ.pop("HARVEST_B200_CONTOUR_BLOCKS", None)
        else:
            os.environ["HARVEST_B200_CONTOUR_BLOCKS"] = saved
