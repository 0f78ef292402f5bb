"""Seeded synthetic test signals for the Harvest workloads.

Every generator returns float64 NumPy arrays and is deterministic for a given
seed. The shapes follow the five benchmark workloads of the engine:

* ``glide_clip``: one voiced glide with unvoiced noise at both ends (the 3 s
  16 kHz clip; also the generator behind the batched and gradient workloads).
* ``segmented_clip``: alternating vibrato-voiced and pink-noise segments (the
  60 s 44.1 kHz clip).
* ``ragged_batch``: many clips of uniformly random length packed ragged.
* ``kind_clip``: the short signal kinds used by the compatibility tests
  (speechlike, low, high, noise, silence).
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "glide_clip", "segmented_clip", "kind_clip", "ragged_batch", "pack",
    "workload",
]


def _harmonics(phase, count, rng, rolloff=1.0):
    out = np.zeros_like(phase)
    offsets = rng.uniform(0, 2 * np.pi, count)
    for k in range(1, count + 1):
        out += np.sin(k * phase + offsets[k - 1]) / k**rolloff
    return out


def glide_clip(seconds=3.0, fs=16000, f0_start=100.0, f0_end=250.0, harmonics=10,
               snr_db=20.0, edge=0.3, seed=0):
    """A linear F0 glide with ``harmonics`` partials of amplitude 1/k and random
    phases, white noise at ``snr_db`` and ``edge`` seconds of noise only at
    each end. Returns ``(x, true_f0)``; ``true_f0(t)`` gives the glide in Hz
    (0 in the unvoiced ends)."""
    rng = np.random.default_rng(seed)
    n = int(round(seconds * fs))
    t = np.arange(n) / fs
    f0 = f0_start + (f0_end - f0_start) * t / max(seconds, 1e-9)
    phase = 2 * np.pi * np.cumsum(f0) / fs
    voiced = _harmonics(phase, harmonics, rng)
    mask = (t >= edge) & (t < seconds - edge)
    ramp = np.clip(np.minimum(t - edge, seconds - edge - t) / 0.01, 0, 1)
    voiced *= mask * ramp
    power = np.mean(voiced[mask] ** 2) if mask.any() else 1.0
    noise = rng.normal(0, np.sqrt(power / 10 ** (snr_db / 10)), n)
    x = np.ascontiguousarray(0.1 * (voiced + noise))

    def true_f0(times):
        times = np.asarray(times, dtype=np.float64)
        g = f0_start + (f0_end - f0_start) * times / max(seconds, 1e-9)
        return np.where((times >= edge) & (times < seconds - edge), g, 0.0)

    return x, true_f0


def _pink(n, rng):
    white = rng.normal(0, 1, n)
    spectrum = np.fft.rfft(white)
    freq = np.arange(len(spectrum))
    freq[0] = 1
    pink = np.fft.irfft(spectrum / np.sqrt(freq), n)
    return pink / (np.std(pink) + 1e-12)


def segmented_clip(seconds=60.0, fs=44100, f0_range=(80.0, 400.0), harmonics=20,
                   voiced_range=(0.2, 1.5), unvoiced_range=(0.1, 0.8), snr_db=30.0,
                   vibrato_hz=5.5, vibrato_depth=0.03, seed=0):
    """Voiced segments (uniform duration, uniform base F0, sinusoidal vibrato,
    ``harmonics`` partials of amplitude 1/k) alternating with pink-noise
    unvoiced segments, plus white noise at ``snr_db``."""
    rng = np.random.default_rng(seed)
    n = int(round(seconds * fs))
    x = np.zeros(n)
    pos, voiced_turn = 0, True
    while pos < n:
        span = rng.uniform(*(voiced_range if voiced_turn else unvoiced_range))
        m = min(n - pos, max(1, int(span * fs)))
        t = np.arange(m) / fs
        if voiced_turn:
            base = rng.uniform(*f0_range)
            f0 = base * (1 + vibrato_depth * np.sin(2 * np.pi * vibrato_hz * t))
            phase = 2 * np.pi * np.cumsum(f0) / fs
            seg = _harmonics(phase, harmonics, rng)
            ramp = np.clip(np.minimum(t, t[-1] - t) / 0.01, 0, 1)
            x[pos:pos + m] = seg * ramp
        else:
            x[pos:pos + m] = 0.3 * _pink(m, rng)
        pos += m
        voiced_turn = not voiced_turn
    power = np.mean(x ** 2) + 1e-12
    x += rng.normal(0, np.sqrt(power / 10 ** (snr_db / 10)), n)
    return np.ascontiguousarray(0.1 * x)


def kind_clip(kind="speechlike", seconds=1.0, fs=24000, seed=1234):
    """Short compatibility-test signals: ``silence`` (zeros), ``noise``
    (white), ``low`` (~80 Hz), ``high`` (~650 Hz) and ``speechlike``
    (intermittent voicing with a wandering 115-205 Hz F0)."""
    rng = np.random.default_rng(seed)
    n = int(round(seconds * fs))
    t = np.arange(n) / fs
    if kind == "silence":
        return np.zeros(n)
    if kind == "noise":
        return rng.normal(0, 0.05, n)
    if kind == "low":
        f0 = 80 + 5 * np.sin(2 * np.pi * 2 * t)
    elif kind == "high":
        f0 = 650 + 30 * np.sin(2 * np.pi * 3 * t)
    elif kind == "speechlike":
        f0 = 160 + 45 * np.sin(2 * np.pi * 0.7 * t) + 3 * np.sin(2 * np.pi * 5 * t)
    else:
        raise ValueError(f"unknown kind {kind!r}")
    phase = 2 * np.pi * np.cumsum(f0) / fs
    x = _harmonics(phase, 10, rng, rolloff=1.3)
    env = np.minimum(1, t / 0.02) * np.minimum(1, (seconds - t) / 0.02)
    if kind == "speechlike":
        env = env * np.clip(8 * np.sin(2 * np.pi * 1.8 * t), 0, 1)
    return np.ascontiguousarray(0.2 * x * env + rng.normal(0, 0.0002, n))


def pack(clips):
    """Pack a list of 1-D arrays into one contiguous buffer plus int64
    offsets of length ``len(clips) + 1``."""
    offsets = np.zeros(len(clips) + 1, dtype=np.int64)
    offsets[1:] = np.cumsum([len(c) for c in clips])
    packed = np.empty(int(offsets[-1]), dtype=np.float64)
    for c, a, b in zip(clips, offsets[:-1], offsets[1:]):
        packed[a:b] = c
    return packed, offsets


def ragged_batch(count=256, fs=16000, seconds=(1.0, 12.0), f0_range=None,
                 snr_range=None, seed=0):
    """``count`` glide clips with uniformly random lengths. ``f0_range`` draws
    a base F0 per clip (the glide spans base..min(2.5 base, 750 Hz));
    ``snr_range`` draws an SNR per clip. Returns ``(clips, true_f0s)``."""
    rng = np.random.default_rng(seed)
    clips, truths = [], []
    for i in range(count):
        length = rng.uniform(*seconds)
        if f0_range is None:
            start, end = 100.0, 250.0
        else:
            start = rng.uniform(*f0_range)
            end = min(2.5 * start, 750.0)
        snr = 20.0 if snr_range is None else rng.uniform(*snr_range)
        x, truth = glide_clip(length, fs, start, end, snr_db=snr,
                              seed=int(rng.integers(1 << 31)))
        clips.append(x)
        truths.append(truth)
    return clips, truths


def workload(name, seed=0):
    """The five benchmark workloads by name. Returns a dict with ``clips``,
    ``fs``, ``f0_floor``, ``f0_ceil``, ``frame_period`` and, for the glide
    workloads, ``truths``."""
    if name == "clip3s_16k":
        x, truth = glide_clip(3.0, 16000, seed=seed)
        return dict(clips=[x], truths=[truth], fs=16000, f0_floor=71.0, f0_ceil=800.0,
                    frame_period=5.0)
    if name == "clip60s_44k":
        return dict(clips=[segmented_clip(60.0, 44100, seed=seed)], fs=44100,
                    f0_floor=71.0, f0_ceil=800.0, frame_period=5.0)
    if name == "batch256_16k":
        clips, truths = ragged_batch(256, 16000, (1.0, 12.0), seed=seed)
        return dict(clips=clips, truths=truths, fs=16000, f0_floor=50.0, f0_ceil=1100.0,
                    frame_period=5.0)
    if name == "batch64_48k":
        clips, truths = ragged_batch(64, 48000, (2.0, 30.0), f0_range=(60.0, 600.0),
                                     snr_range=(0.0, 20.0), seed=seed)
        return dict(clips=clips, truths=truths, fs=48000, f0_floor=71.0, f0_ceil=800.0,
                    frame_period=1.0)
    if name == "grad32x4s_16k":
        clips, truths = ragged_batch(32, 16000, (4.0, 4.0), seed=seed)
        return dict(clips=clips, truths=truths, fs=16000, f0_floor=71.0, f0_ceil=800.0,
                    frame_period=5.0)
    raise ValueError(f"unknown workload {name!r}")
