"""The dense FP64 torch restatement used to check the F0 gradient, checked on
CPU against the C checker: its forward pass must rebuild the checker's
step-3/step-4 contours, smoothed contour and output F0 from a tape, and its
autograd gradient must match central finite differences of the checker's
own Harvest (eps 1e-6) wherever Harvest is smooth."""
import numpy as np
import pytest
import torch

import oracle
from harvest_cuda_b200 import signals
from tests import torch_reference as ref

CASES = [
    ("glide16k", lambda: signals.glide_clip(0.6, 16000, edge=0.1, seed=3)[0], 16000),
    ("speech44k", lambda: signals.kind_clip("speechlike", 0.35, 44100), 44100),
]


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    scale = np.maximum(np.abs(b), 1e-300)
    return float(np.max(np.where((a == 0) & (b == 0), 0.0, np.abs(a - b) / scale)))


@pytest.mark.parametrize("name,make,fs", CASES, ids=[c[0] for c in CASES])
def test_reference_rebuilds_checker_contours(name, make, fs):
    x = make()
    checker = oracle.best()
    st = checker.stages(x, fs)
    tape = ref.tape_from_stages(st)
    assert (tape[:, 0] > 0).sum() > 20, "the case must have voiced frames"
    f0, mid = ref.harvest_from_tape(torch.from_numpy(x), fs, tape)
    voiced = tape[:, 0] > 0
    assert _rel(mid["s3"].numpy()[voiced], tape[voiced, 0]) < 1e-12
    assert _rel(mid["s4"].numpy(), st["fixed"]) < 1e-12
    np.testing.assert_allclose(mid["smoothed"].numpy(), st["smoothed"], rtol=1e-11, atol=0)
    np.testing.assert_allclose(f0.detach().numpy(), checker.harvest(x, fs)[0], rtol=1e-11, atol=0)


def test_reference_gradient_matches_checker_differences():
    x = signals.glide_clip(0.6, 16000, edge=0.1, seed=3)[0]
    fs, eps = 16000, 1e-6
    checker = oracle.best()
    tape = ref.tape_from_stages(checker.stages(x, fs))
    base = checker.harvest(x, fs)[0]
    rng = np.random.default_rng(0)
    weights = rng.normal(size=base.size) * (base > 0)
    xt = torch.from_numpy(x.copy()).requires_grad_(True)
    f0, _ = ref.harvest_from_tape(xt, fs, tape)
    (f0 * torch.from_numpy(weights)).sum().backward()
    grad = xt.grad.numpy()
    positions = rng.choice(np.arange(int(0.15 * fs), int(0.45 * fs)), 12, replace=False)
    checked = 0
    for m in positions:
        values = []
        for step in (eps, -eps):
            xp = x.copy()
            xp[m] += step
            values.append(checker.harvest(xp, fs)[0])
        up, down = values
        if not (np.array_equal(up > 0, base > 0) and np.array_equal(down > 0, base > 0)):
            continue   # a voicing decision flipped: no derivative here
        fwd = weights @ (up - base) / eps
        bwd = weights @ (base - down) / eps
        central = weights @ (up - down) / (2 * eps)
        if abs(fwd - bwd) > 1e-3 * max(abs(central), 1e-3):
            continue   # a candidate choice switched inside the step
        assert abs(grad[m] - central) <= 1e-5 * max(abs(central), 1e-2 * np.abs(grad).max()), (m, grad[m], central)
        checked += 1
    assert checked >= 10
