"""Dense FP64 PyTorch restatement of the smooth part of Harvest, used to
check the engine's F0 gradient. Test infrastructure only.

Harvest's output F0 is piecewise smooth in the waveform. Given a clip and the
tape of a forward pass (per 1 ms frame: the FixF0Contour step-3 F0 and the
initial candidate F0 it was refined from), this module rebuilds the output F0
from differentiable torch operations, following the reference's bundled
WORLD Harvest (file:line in WORLD's src/):

* decimation, GetWaveformAndSpectrumSub + decimate (harvest.cpp:43-66,
  matlabfunctions.cpp:178-204), with FilterForDecimate's order-3 low-pass
  (matlabfunctions.cpp:27-124) applied as a causal convolution with its
  impulse response, truncated below 1e-30 of its peak;
* the DC removal of GetWaveformAndSpectrum (harvest.cpp:82-86);
* GetRefinedF0 + FixF0 (harvest.cpp:434-617) for the tape's candidate of
  every voiced frame, with the two windowed spectra evaluated as dense DFTs
  at the harmonic bins;
* FixStep4 (harvest.cpp:1000-1022), SmoothF0Contour + FilteringF0
  (harvest.cpp:1049-1113, the Butterworth filter again as a convolution),
  and the nearest-frame resampling of Harvest (harvest.cpp:1246-1251).

torch.autograd through it gives dL/dx with every discrete choice held at the
tape's values, which is what the engine's adjoint kernels compute.
"""
from __future__ import annotations

import math

import numpy as np
import torch
import torch.nn.functional as nnf

# FilterForDecimate (matlabfunctions.cpp:27-113): a[0..2], b[0..1] by ratio.
_LOW = {
    2: ((0.041156734567757189, -0.42599112459189636, 0.041037215479961225),
        (0.16797464681802227, 0.50392394045406674)),
    3: ((0.95039378983237421, -0.67429146741526791, 0.15412211621346475),
        (0.071221945171178636, 0.21366583551353591)),
    4: ((1.4499664446880227, -0.98943497080950582, 0.24578252340690215),
        (0.036710750339322612, 0.11013225101796784)),
    5: ((1.7610939654280557, -1.2554914843859768, 0.3237186507788215),
        (0.021334858522387423, 0.06400457556716227)),
    6: ((1.9715352749512141, -1.4686795689225347, 0.3893908434965701),
        (0.013469181309343825, 0.040407543928031475)),
}
# FilteringF0 (harvest.cpp:1079-1080).
_BUTTER_B = (0.0078202080334971724, 0.015640416066994345)
_BUTTER_A = (1.7347257688092754, -0.76600660094326412)
_LAG = 300


def ratio_for(fs):
    v = fs / 8000.0
    r = int(v + 0.5) if v > 0 else int(v - 0.5)
    return min(12, max(1, r))


def round_away(v):
    return int(v + 0.5) if v > 0 else int(v - 0.5)


def _impulse(step, limit=1e-30, length=1 << 16):
    """Impulse response of a recursive filter given as a step function."""
    state = [0.0, 0.0, 0.0]
    h = np.zeros(length)
    for i in range(length):
        h[i] = step(1.0 if i == 0 else 0.0, state)
    keep = np.nonzero(np.abs(h) > limit * np.abs(h).max())[0][-1] + 1
    return torch.from_numpy(h[:keep].copy())


def _lowpass_impulse(r):
    a, b = _LOW[r]

    def step(x, s):
        w = x + a[0] * s[0] + a[1] * s[1] + a[2] * s[2]
        out = b[0] * w + b[1] * s[0] + b[1] * s[1] + b[0] * s[2]
        s[2], s[1], s[0] = s[1], s[0], w
        return out
    return _impulse(step)


def _butter_impulse():
    b, a = _BUTTER_B, _BUTTER_A

    def step(x, s):
        w = x + a[0] * s[0] + a[1] * s[1]
        out = b[0] * w + b[1] * s[0] + b[0] * s[1]
        s[1], s[0] = s[0], w
        return out
    return _impulse(step)


def causal(x, h):
    """y[i] = sum_k h[k] x[i - k] (zero initial state)."""
    return nnf.conv1d(nnf.pad(x.view(1, 1, -1), (h.numel() - 1, 0)), h.flip(0).view(1, 1, -1)).view(-1)


def decimate(x, fs):
    """The decimated, DC-free waveform of Harvest as torch operations."""
    r = ratio_for(fs)
    n = x.numel()
    y_len = math.ceil(n / r)
    if r == 1:
        y = x
    else:
        lag = int(math.ceil(140.0 / r) * r)
        m = n + 2 * lag
        ext = x[torch.clamp(torch.arange(m) - lag, 0, n - 1)]
        i9 = torch.arange(9)
        a = torch.cat([2 * ext[0] - ext[9 - i9], ext, 2 * ext[m - 1] - ext[m - 2 - i9]])
        h = _lowpass_impulse(r)
        a = causal(a, h).flip(0)
        a = causal(a, h).flip(0)
        nout = (m - 1) // r + 1
        nbeg = r - r * nout + m
        y = a[nbeg + (lag // r + torch.arange(y_len)) * r + 8]
    return y - y.sum() / y_len


def refine(y, fs, t, f0c):
    """FixF0's refined F0 of candidate f0c at time t (seconds) of waveform y
    sampled at fs, as a torch scalar."""
    half = int(1.5 * fs / f0c + 1.0)
    length = 2 * half + 1
    span = (2.0 * half + 1.0) / fs
    n = int(2.0 ** (2 + int(math.log(half * 2.0 + 1.0) / 0.69314718055994529)))
    base = round_away((t + (-half) / fs) * fs + 0.001)
    i = np.arange(length)
    tmp = (base + i - 1.0) / fs - t
    w = 0.42 + 0.5 * np.cos(2.0 * np.pi * tmp / span) + 0.08 * np.cos(4.0 * np.pi * tmp / span)
    dw = np.empty(length)
    dw[0] = -w[1] / 2.0
    dw[1:-1] = -(w[2:] - w[:-2]) / 2.0
    dw[-1] = w[-2] / 2.0
    harmonics = min(int(fs / 2.0 / f0c), 6)
    bins = np.array([round_away(f0c * n / fs * (h + 1)) for h in range(harmonics)])
    theta = 2.0 * np.pi * ((bins[:, None] * i[None, :]) % n) / n       # [harmonics, length]
    cos, sin = torch.from_numpy(np.cos(theta)), torch.from_numpy(np.sin(theta))
    seg = y[torch.clamp(torch.arange(length) + base - 1, 0, y.numel() - 1)]
    a = seg * torch.from_numpy(w)
    d = seg * torch.from_numpy(dw)
    mr, mi = cos @ a, -(sin @ a)
    dr, di = cos @ d, -(sin @ d)
    power = mr * mr + mi * mi
    cross = mr * di - mi * dr
    inst = torch.from_numpy(bins * fs / n) + cross / power * fs / 2.0 / math.pi
    amp = torch.sqrt(power)
    order = torch.arange(1, harmonics + 1, dtype=torch.float64)
    return (amp * inst).sum() / ((amp * order).sum() + 1e-12)


def boundary_list(values):
    """GetBoundaryList (harvest.cpp:727-743) of a NumPy array."""
    out, prev, length = [], 0, len(values)
    for i in range(1, length):
        v = 0 if i == length - 1 else int(values[i] > 0)
        if v != prev:
            out.append(i - len(out) % 2)
        prev = v
    return out


def fill_gaps(s3):
    """FixStep4 with threshold 9 (harvest.cpp:1000-1022)."""
    vals = s3.detach().numpy()
    bl = boundary_list(vals)
    parts = list(s3.unbind())
    for i in range(len(bl) // 2 - 1):
        a, b = bl[2 * i + 1], bl[2 * (i + 1)]
        distance = b - a - 1
        if distance >= 9:
            continue
        v0, v1 = s3[a] + 1, s3[b] - 1
        slope = (v1 - v0) / (distance + 1.0)
        for cnt, j in enumerate(range(a + 1, b), start=1):
            parts[j] = v0 + slope * cnt
    return torch.stack(parts)


def smooth(s4):
    """SmoothF0Contour (harvest.cpp:1079-1113)."""
    frames = s4.numel()
    padded = torch.cat([torch.zeros(_LAG, dtype=s4.dtype), s4, torch.zeros(_LAG, dtype=s4.dtype)])
    length = padded.numel()
    bl = boundary_list(padded.detach().numpy())
    h = _butter_impulse()
    out = torch.zeros(frames, dtype=s4.dtype)
    for k in range(len(bl) // 2):
        st, ed = bl[2 * k], bl[2 * k + 1]
        chan = padded[torch.clamp(torch.arange(length), st, ed)]
        res = causal(causal(chan, h).flip(0), h).flip(0)
        out = out.index_copy(0, torch.arange(st - _LAG, ed - _LAG + 1), res[st:ed + 1])
    return out


def resample(smoothed, n, fs, frame_period):
    out_len = int(1000.0 * n / fs / frame_period) + 1
    idx = [min(smoothed.numel() - 1, round_away(i * frame_period / 1000.0 * 1000.0)) for i in range(out_len)]
    return smoothed[torch.tensor(idx)]


def harvest_from_tape(x, fs, tape, frame_period=5.0):
    """Output F0 of one clip (torch, differentiable in x) with the discrete
    choices of `tape` ([frames, 2]: step-3 F0, initial candidate F0).
    Returns (f0, intermediates) where intermediates holds y, s3, s4 and the
    smoothed 1 ms contour."""
    tape = np.asarray(tape, dtype=np.float64).reshape(-1, 2)
    y = decimate(x, fs)
    fs_r = fs / ratio_for(fs)
    parts = []
    for f in range(tape.shape[0]):
        if tape[f, 0] > 0 and tape[f, 1] > 0:
            parts.append(refine(y, fs_r, f * 1 / 1000.0, tape[f, 1]))
        else:
            parts.append(torch.zeros((), dtype=torch.float64))
    s3 = torch.stack(parts)
    s4 = fill_gaps(s3)
    sm = smooth(s4)
    return resample(sm, x.numel(), fs, frame_period), dict(y=y, s3=s3, s4=s4, smoothed=sm)


def tape_from_stages(st):
    """A tape built from a CPU checker's stage dump: a frame of the step-4
    contour that equals one of its pruned candidates carries that value and
    the candidate's initial F0; FixStep4's fills (interpolated values) and
    unvoiced frames carry zeros."""
    fixed, pruned, cand = st["fixed"], st["pruned"], st["cand"]
    columns = 7 * st["count"]
    tape = np.zeros((len(fixed), 2))
    for f, v in enumerate(fixed):
        if v <= 0:
            continue
        hits = np.nonzero(pruned[f, :columns] == v)[0]
        if hits.size:
            tape[f] = (v, cand[f, hits[0]])
    return tape
