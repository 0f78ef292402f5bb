"""The ragged batched path, the workspace cache and concurrency on a GPU
(reference tests/test_compatibility.py:103-227 for the cache and thread
contract; batching has no reference counterpart)."""
from concurrent.futures import ThreadPoolExecutor
from threading import Barrier

import numpy as np
import pytest

import harvest_cuda_b200 as hv
from harvest_cuda_b200 import signals
from harvest_cuda_b200.metrics import compare

pytestmark = pytest.mark.gpu


def _clips(count=12, fs=16000, seed=5):
    clips, _ = signals.ragged_batch(count, fs, (0.3, 2.5), seed=seed)
    return clips


def test_batch_equals_per_clip(gpu):
    clips = _clips()
    batch = hv.harvest_many(clips, 16000, 50.0, 1100.0, 5.0)
    for x, (f0, t) in zip(clips, batch):
        single = hv.harvest(x, 16000, 50.0, 1100.0, 5.0)
        np.testing.assert_array_equal(f0, single[0])
        np.testing.assert_array_equal(t, single[1])


def test_batch_graph_and_stagewise_agree(gpu):
    clips = _clips(seed=9)
    packed, off = signals.pack(clips)
    a = hv.harvest_batch(packed, off, 16000)
    b = hv.harvest_batch(packed, off, 16000, graph=False)
    c = hv.harvest_batch(packed, off, 16000)   # graph replay
    for u, v in zip(a, b):
        np.testing.assert_array_equal(u, v)
    for u, v in zip(a, c):
        np.testing.assert_array_equal(u, v)


def test_contour_block_size_does_not_change_f0(gpu):
    # A batch with at least as many clips as the GPU has SMs (148 on a B200)
    # runs the contour's last kernel with 256 threads per clip, a smaller one
    # with 512; both must give the same F0 for every clip.
    clips, _ = signals.ragged_batch(200, 16000, (0.3, 1.2), seed=21)
    big = hv.harvest_many(clips, 16000, 50.0, 1100.0, 5.0)
    small = hv.harvest_many(clips[:9], 16000, 50.0, 1100.0, 5.0)
    for (f0, t), (g0, u) in zip(big[:9], small):
        np.testing.assert_array_equal(f0, g0)
        np.testing.assert_array_equal(t, u)


def test_batch_matches_checker(gpu, checker):
    clips = _clips(count=6, seed=11)
    out = hv.harvest_many(clips, 16000, 50.0, 1100.0, 5.0)
    for x, (f0, t) in zip(clips, out):
        rf, rt = checker.harvest(x, 16000, 50.0, 1100.0, 5.0)
        np.testing.assert_array_equal(t, rt)
        m = compare(rf, f0)
        assert m["vuv_disagreement"] <= 0.001
        if m["joint_voiced_frames"]:
            assert m["rel_max"] <= 1e-6


def test_batch_shapes_change_and_return(gpu):
    # New batch shapes build new plans; returning to an earlier one reuses it.
    first = _clips(4, seed=1)
    second = _clips(7, 24000, seed=2)
    a = hv.harvest_many(first, 16000)
    hv.harvest_many(second, 24000, 65.0, 900.0, 2.5)
    b = hv.harvest_many(first, 16000)
    for (f0a, ta), (f0b, tb) in zip(a, b):
        np.testing.assert_array_equal(f0a, f0b)
        np.testing.assert_array_equal(ta, tb)


def test_mixed_short_and_long_clips(gpu, checker):
    clips = [np.zeros(6 * 2), signals.kind_clip("high", 0.2, 16000),
             signals.kind_clip("speechlike", 3.0, 16000), np.zeros(240)]
    out = hv.harvest_many(clips, 16000)
    for x, (f0, t) in zip(clips, out):
        rf, rt = checker.harvest(x, 16000)
        np.testing.assert_array_equal(t, rt)
        np.testing.assert_allclose(f0, rf, rtol=1e-7, atol=1e-5)


def test_clear_cache_preserves_outputs_and_other_threads(gpu):
    x = signals.kind_clip("speechlike", 0.7, 24000)
    expected = hv.harvest(x, 24000)
    saved = tuple(a.copy() for a in expected)
    ready = Barrier(2)

    def worker():
        before = hv.harvest(x, 24000)
        ready.wait(timeout=60)
        ready.wait(timeout=60)
        after = hv.harvest(x, 24000)
        hv.clear_cache()
        return before, after

    with ThreadPoolExecutor(max_workers=1) as pool:
        future = pool.submit(worker)
        ready.wait(timeout=60)
        hv.clear_cache()
        hv.clear_cache()
        ready.wait(timeout=60)
        actual = [*future.result(), hv.harvest(x, 24000)]
    hv.clear_cache()
    for result in [expected, *actual]:
        for got, want in zip(result, saved):
            np.testing.assert_array_equal(got, want)


def test_concurrent_calls(gpu, checker):
    inputs = [(signals.kind_clip("speechlike", 0.3, 16000), 16000),
              (signals.kind_clip("high", 0.5, 24000), 24000)] * 3
    with ThreadPoolExecutor(max_workers=3) as pool:
        futures = [pool.submit(hv.harvest, x, fs) for x, fs in inputs]
        pool.submit(hv.clear_cache).result()
        results = [f.result() for f in futures]
    for (x, fs), (f0, t) in zip(inputs, results):
        rf, rt = checker.harvest(x, fs)
        np.testing.assert_array_equal(t, rt)
        np.testing.assert_allclose(f0, rf, rtol=1e-7, atol=1e-5)


def test_explicit_device_and_out_of_range(gpu):
    x = signals.kind_clip("speechlike", 0.35, 16000)
    expected = hv.harvest(x, 16000)
    assert hv.cuda_available(device=0)
    assert not hv.cuda_available(device=2**31 - 1)
    with pytest.raises(ValueError, match="out of range"):
        hv.harvest(x, 16000, device=2**31 - 1)
    actual = hv.harvest(x, 16000, device=0)
    for got, want in zip(actual, expected):
        np.testing.assert_array_equal(got, want)
    f0, t, stages = hv.profile(x, 16000)
    np.testing.assert_array_equal(f0, expected[0])
    assert set(stages) == {"decimate", "band_bank", "candidates", "refine", "prune", "contour"}
    assert all(np.isfinite(v) and v >= 0 for v in stages.values())
