"""BatchPipeline: host batches with uploads and downloads overlapped across
consecutive batches. Its results must equal harvest_batch's bit for bit,
whatever the order of submit and result calls, batch shapes and input
memory kinds."""
import numpy as np
import pytest

import harvest_cuda_b200 as hv
from harvest_cuda_b200 import signals

pytestmark = pytest.mark.gpu


def _batch(seconds, fs, seed):
    clips = [signals.glide_clip(s, fs, seed=seed + i)[0] for i, s in enumerate(seconds)]
    return signals.pack(clips)


def test_matches_harvest_batch_across_shapes_and_memory_kinds(gpu):
    import torch
    from harvest_cuda_b200.pipeline import BatchPipeline
    batches = [_batch((1.2, 0.6, 2.1), 16000, 0), _batch((0.9,), 16000, 5), _batch((2.5, 0.4, 1.0, 1.7), 16000, 9)]
    # Pinned input (uploaded directly), plain NumPy (staged), read-only (staged).
    pinned = torch.from_numpy(batches[0][0]).pin_memory().numpy()
    readonly = batches[2][0].copy()
    readonly.setflags(write=False)
    inputs = [(pinned, batches[0][1]), batches[1], (readonly, batches[2][1])]
    want = [hv.harvest_batch(x, o, 16000, 50.0, 1100.0, 5.0) for x, o in batches]
    pipe = BatchPipeline(16000, 50.0, 1100.0, 5.0, depth=2)
    got = []
    pipe.submit(*inputs[0])
    pipe.submit(*inputs[1])
    with pytest.raises(RuntimeError):
        pipe.submit(*inputs[2])
    got.append(pipe.result())
    pipe.submit(*inputs[2])
    got.append(pipe.result())
    got.append(pipe.result())
    assert pipe.pending() == 0
    for g, w in zip(got, want):
        for a, b in zip(g, w):
            assert np.array_equal(a, b)
    # A second round reuses the slots (same and different shapes).
    for x, o in (inputs[2], inputs[0], inputs[2]):
        pipe.submit(x, o)
        if pipe.pending() == pipe.depth:
            pipe.result()
    last = None
    while pipe.pending():
        last = pipe.result()
    for a, b in zip(last, want[2]):
        assert np.array_equal(a, b)


def test_non_finite_batch_raises_at_result_and_pipeline_continues(gpu):
    from harvest_cuda_b200.pipeline import BatchPipeline
    x, o = _batch((0.8, 1.1), 16000, 3)
    bad = x.copy()
    bad[int(o[1]) + 10] = np.nan
    pipe = BatchPipeline(16000, depth=3)
    pipe.submit(x, o)
    pipe.submit(bad, o)
    pipe.submit(x, o)
    want = hv.harvest_batch(x, o, 16000)
    first = pipe.result()
    with pytest.raises(ValueError, match="finite"):
        pipe.result()
    third = pipe.result()
    for g in (first, third):
        for a, b in zip(g, want):
            assert np.array_equal(a, b)


def test_rejects_bad_batches(gpu):
    from harvest_cuda_b200.pipeline import BatchPipeline
    x, o = _batch((0.5,), 16000, 1)
    pipe = BatchPipeline(16000)
    with pytest.raises(ValueError):
        pipe.submit(x, [0, x.size + 1])
    with pytest.raises(ValueError, match="empty"):
        pipe.submit(x, [0, 0, x.size])
    with pytest.raises(TypeError):
        pipe.submit(x.astype(np.float32), o)
    with pytest.raises(RuntimeError):
        pipe.result()
