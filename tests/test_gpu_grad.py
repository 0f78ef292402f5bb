"""The F0 gradient on the GPU: hv_harvest_grad_forward / _backward through
harvest_cuda_b200.autograd, checked against

* the dense FP64 torch restatement (tests/torch_reference.py) driven by the
  GPU forward pass's own tape, on two clips;
* central finite differences (eps 1e-6) of the GPU forward pass at random
  samples of 4 s clips of the gradient workload's generator, with
  L = sum over voiced frames of (f0 - true f0)^2.
"""
import ctypes as ct

import numpy as np
import pytest

import harvest_cuda_b200 as hv
from harvest_cuda_b200 import _native, autograd, signals
from tests import torch_reference as ref

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _forward_tape(clips, fs, f0_floor=71.0, f0_ceil=800.0, period=5.0):
    """f0 and tape of the GPU forward pass, through the C ABI."""
    torch = _torch()
    offsets = np.concatenate([[0], np.cumsum([len(c) for c in clips])]).astype(np.int64)
    x = torch.from_numpy(np.concatenate(clips)).cuda()
    outs = sum(hv.output_length(len(c), fs, period) for c in clips)
    frames = sum(hv.output_length(len(c), fs, 1.0) for c in clips)
    f0 = torch.empty(outs, dtype=torch.float64, device="cuda")
    tape = torch.empty(2 * frames, dtype=torch.float64, device="cuda")
    status = _native.lib.hv_harvest_grad_forward(
        x.data_ptr(), offsets.ctypes.data_as(ct.POINTER(ct.c_int64)), len(clips), fs, f0_floor, f0_ceil,
        period, 0, f0.data_ptr(), None, tape.data_ptr(), None)
    _native.raise_for(status)
    torch.cuda.synchronize()
    return f0.cpu().numpy(), tape.cpu().numpy().reshape(-1, 2)


def _loss(f0, times, true_f0):
    """L = sum over voiced frames of (f0 - true f0)^2."""
    torch = _torch()
    target = torch.as_tensor(true_f0(times.detach().cpu().numpy()), device=f0.device)
    voiced = (f0.detach() > 0) & (target > 0)
    return ((f0 - target) ** 2 * voiced).sum()


def test_forward_is_the_regular_path(gpu):
    torch = _torch()
    clips = [signals.glide_clip(1.3, 16000, seed=s)[0] for s in (1, 2, 3)]
    got = autograd.harvest_f0([torch.from_numpy(c).cuda() for c in clips], 16000)
    want = hv.harvest_many(clips, 16000)
    for (f0, t), (wf, wt) in zip(got, want):
        assert np.array_equal(f0.detach().cpu().numpy(), wf)
        assert np.array_equal(t.cpu().numpy(), wt)


def test_tape_matches_checker(gpu, checker):
    x = signals.glide_clip(1.0, 16000, edge=0.15, seed=7)[0]
    _, tape = _forward_tape([x], 16000)
    want = ref.tape_from_stages(checker.stages(x, 16000))
    both = (tape[:, 0] > 0) & (want[:, 0] > 0)
    assert both.sum() > 0.99 * max((tape[:, 0] > 0).sum(), (want[:, 0] > 0).sum())
    np.testing.assert_allclose(tape[both, 0], want[both, 0], rtol=1e-9, atol=0)
    assert np.all(tape[tape[:, 0] > 0, 1] > 0)


# The longer clips hold voiced sections of more than 1024 frames, whose
# smoothing adjoint the whole warp runs in chunks.
@pytest.mark.parametrize("fs,seconds", [(16000, 0.9), (44100, 0.6), (16000, 1.8), (44100, 1.4)])
def test_gradient_matches_torch_reference(gpu, fs, seconds):
    torch = _torch()
    made = [signals.glide_clip(seconds, fs, edge=0.15, seed=s) for s in (11, 12)]
    clips = [m[0] for m in made]
    xs = [torch.from_numpy(c).cuda().requires_grad_(True) for c in clips]
    out = autograd.harvest_f0(xs, fs)
    loss = sum(_loss(f0, t, m[1]) for (f0, t), m in zip(out, made))
    loss.backward()
    _, tape = _forward_tape(clips, fs)
    row = 0
    for c, (x, (f0, t), m) in enumerate(zip(xs, out, made)):
        frames = hv.output_length(len(clips[c]), fs, 1.0)
        xr = torch.from_numpy(clips[c].copy()).requires_grad_(True)
        f0r, _ = ref.harvest_from_tape(xr, fs, tape[row:row + frames])
        row += frames
        np.testing.assert_allclose(f0r.detach().numpy(), f0.detach().cpu().numpy(), rtol=1e-11, atol=0)
        _loss(f0r, t.cpu(), m[1]).backward()
        got, want = x.grad.cpu().numpy(), xr.grad.numpy()
        assert np.abs(want).max() > 0
        assert np.abs(got - want).max() <= 1e-9 * np.abs(want).max()


def test_gradient_matches_finite_differences(gpu):
    """Central differences at eps 1e-6 (and, more sharply, 1e-5) against dL/dx
    at random samples. The F0 values carry rounding noise near one unit in
    the last place; divided by 2 eps it makes about 1e-6 of absolute noise in
    a difference at eps 1e-6 (falling as 1/eps), so errors are measured
    against the gradient's scale, max |dL/dx| over the clip."""
    torch = _torch()
    fs, per_clip = 16000, 16
    made = [signals.glide_clip(4.0, fs, seed=20 + s) for s in range(4)]
    clips = [m[0] for m in made]
    xs = [torch.from_numpy(c).cuda().requires_grad_(True) for c in clips]
    out = autograd.harvest_f0(xs, fs)
    sum(_loss(f0, t, m[1]) for (f0, t), m in zip(out, made)).backward()
    rng = np.random.default_rng(5)
    worst = {1e-6: 0.0, 1e-5: 0.0}
    skipped = 0
    for c, (x, m) in enumerate(zip(clips, made)):
        grad = xs[c].grad.cpu().numpy()
        scale = np.abs(grad).max()
        base_f0, times = out[c][0].detach().cpu().numpy(), out[c][1].cpu().numpy()
        target = m[1](times)
        voiced = (base_f0 > 0) & (target > 0)
        positions = rng.choice(len(x), per_clip, replace=False)
        batch = []
        for p in positions:
            for step in (1e-6, -1e-6, 1e-5, -1e-5):
                xp = x.copy()
                xp[p] += step
                batch.append(xp)
        results = hv.harvest_many(batch, fs)
        for k, p in enumerate(positions):
            for j, eps in enumerate((1e-6, 1e-5)):
                up, down = results[4 * k + 2 * j][0], results[4 * k + 2 * j + 1][0]
                if not (np.array_equal(up > 0, base_f0 > 0) and np.array_equal(down > 0, base_f0 > 0)):
                    skipped += 1
                    continue
                # Differences of L formed frame by frame, (a - t)^2 - (b - t)^2 =
                # (a - b)(a + b - 2t), so that no sum of large terms cancels.
                central = np.sum(((up - down) * (up + down - 2 * target))[voiced]) / (2 * eps)
                curvature = np.sum(((up - base_f0) * (up + base_f0 - 2 * target) -
                                    (base_f0 - down) * (base_f0 + down - 2 * target))[voiced]) / eps
                if abs(curvature) > 1e-3 * max(abs(central), 1.0):
                    skipped += 1       # a discrete choice switched inside the step
                    continue
                worst[eps] = max(worst[eps], abs(grad[p] - central) / scale)
    assert skipped <= 4
    assert worst[1e-6] <= 1e-5, worst
    assert worst[1e-5] <= 1e-6, worst


def test_gradient_relative_error_where_it_is_large(gpu):
    """Per sample, where the gradient is large: at 12 samples drawn from each
    clip's 200 largest |dL/dx|, the central difference at eps 1e-5 agrees
    with dL/dx within 1e-5 relative to that sample's own value (there the
    difference noise, about 1e-7 of the clip's max |dL/dx|, is far below it)."""
    torch = _torch()
    fs, per_clip, eps = 16000, 12, 1e-5
    made = [signals.glide_clip(4.0, fs, seed=40 + s) for s in range(4)]
    clips = [m[0] for m in made]
    xs = [torch.from_numpy(c).cuda().requires_grad_(True) for c in clips]
    out = autograd.harvest_f0(xs, fs)
    sum(_loss(f0, t, m[1]) for (f0, t), m in zip(out, made)).backward()
    rng = np.random.default_rng(11)
    worst, checked, skipped = 0.0, 0, 0
    for c, (x, m) in enumerate(zip(clips, made)):
        grad = xs[c].grad.cpu().numpy()
        base_f0, times = out[c][0].detach().cpu().numpy(), out[c][1].cpu().numpy()
        target = m[1](times)
        voiced = (base_f0 > 0) & (target > 0)
        positions = rng.choice(np.argsort(-np.abs(grad))[:200], per_clip, replace=False)
        batch = []
        for p in positions:
            for step in (eps, -eps):
                xp = x.copy()
                xp[p] += step
                batch.append(xp)
        results = hv.harvest_many(batch, fs)
        for k, p in enumerate(positions):
            up, down = results[2 * k][0], results[2 * k + 1][0]
            if not (np.array_equal(up > 0, base_f0 > 0) and np.array_equal(down > 0, base_f0 > 0)):
                skipped += 1
                continue
            central = np.sum(((up - down) * (up + down - 2 * target))[voiced]) / (2 * eps)
            curvature = np.sum(((up - base_f0) * (up + base_f0 - 2 * target) -
                                (base_f0 - down) * (base_f0 + down - 2 * target))[voiced]) / eps
            if abs(curvature) > 1e-3 * max(abs(central), 1.0):
                skipped += 1       # a discrete choice switched inside the step
                continue
            worst = max(worst, abs(grad[p] - central) / abs(grad[p]))
            checked += 1
    # Large gradients sit where F0 is most sensitive, so a step there more
    # often switches a discrete choice; those samples are skipped.
    assert checked >= 24, (checked, skipped)
    assert worst <= 1e-5, worst


def test_raw_candidates_forward_is_the_pipelines(gpu):
    torch = _torch()
    x = signals.glide_clip(1.2, 16000, seed=4)[0]
    raw = autograd.raw_candidates(torch.from_numpy(x).cuda(), 16000).cpu().numpy()
    want = hv.api.stages(x, 16000)["raw"]
    assert raw.shape == want.shape
    assert np.array_equal(raw, want)


def test_raw_candidate_gradient_matches_finite_differences(gpu):
    """The band-bank adjoint (per-band candidates) against central
    differences of the forward pass, at eps 1e-6 and 1e-5, errors measured
    against the gradient's scale as for the F0 gradient."""
    torch = _torch()
    fs, per_clip = 16000, 12
    x = signals.glide_clip(1.5, fs, seed=31)[0]
    xt = torch.from_numpy(x.copy()).cuda().requires_grad_(True)
    raw = autograd.raw_candidates(xt, fs)
    mask = (raw.detach() != 0)
    rng = np.random.default_rng(8)
    weights = torch.from_numpy(rng.normal(size=tuple(raw.shape))).cuda() * mask
    (raw * weights).sum().backward()
    grad = xt.grad.cpu().numpy()
    scale = np.abs(grad).max()
    assert scale > 0
    w = weights.cpu().numpy()
    base = raw.detach().cpu().numpy()
    positions = rng.choice(np.arange(int(0.3 * fs), int(1.2 * fs)), per_clip, replace=False)
    worst = {1e-6: 0.0, 1e-5: 0.0}
    skipped = 0
    for eps in (1e-6, 1e-5):
        batch = []
        for p in positions:
            for step in (eps, -eps):
                xp = x.copy()
                xp[p] += step
                batch.append(torch.from_numpy(xp).cuda())
        outs = [r.cpu().numpy() for r in autograd.raw_candidates(batch, fs)]
        for k, p in enumerate(positions):
            up, down = outs[2 * k], outs[2 * k + 1]
            if not (np.array_equal(up != 0, base != 0) and np.array_equal(down != 0, base != 0)):
                skipped += 1
                continue
            central = np.sum((up - down) * w) / (2 * eps)
            curvature = np.sum((up - 2 * base + down) * w) / eps
            if abs(curvature) > 1e-3 * max(abs(central), scale * 1e-3):
                skipped += 1
                continue
            worst[eps] = max(worst[eps], abs(grad[p] - central) / scale)
    assert skipped <= 6, skipped
    assert worst[1e-6] <= 1e-5, worst
    assert worst[1e-5] <= 1e-6, worst
