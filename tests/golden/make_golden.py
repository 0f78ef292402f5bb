"""Regenerates the golden fixtures in this directory from the reference's own
bundled WORLD Harvest (oracle/_ref/libworld_ref.so, built by oracle/Makefile
from the reference sources).

Each fixture stores the input clip and WORLD's (f0, times) for it; index.json
lists them with their settings. Run from the repository root:

    python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from harvest_cuda_b200 import signals  # noqa: E402


def quirk_clip(length, fs=8000):
    # Excites the two spectrum bins that WORLD's band filter overwrites
    # (Nyquist and n/2 - 1 of the whole-signal FFT, n = 32768 here).
    x = signals.kind_clip("speechlike", length / fs, fs)
    i = np.arange(x.size)
    return x + 0.01 * ((1 - 2 * (i % 2)) + np.cos(2 * np.pi * (0.5 - 1 / 32768) * i))


def cases():
    yield "speech_16k_p5", signals.kind_clip("speechlike", 0.7, 16000), 16000, 71.0, 800.0, 5.0
    yield "speech_8k_p1", signals.kind_clip("speechlike", 0.5, 8000), 8000, 71.0, 800.0, 1.0
    yield "high_24k_p2_5", signals.kind_clip("high", 0.5, 24000), 24000, 71.0, 800.0, 2.5
    yield "low_44k_p10", signals.kind_clip("low", 0.4, 44100), 44100, 71.0, 800.0, 10.0
    yield "noise_48k_p5", signals.kind_clip("noise", 0.3, 48000), 48000, 71.0, 800.0, 5.0
    yield "silence_24k_240", np.zeros(240), 24000, 71.0, 800.0, 5.0
    yield "glide_16k_50_1100", signals.glide_clip(1.0, 16000, seed=3)[0], 16000, 50.0, 1100.0, 5.0
    yield "quirk_8k_24577", quirk_clip(24577), 8000, 71.0, 800.0, 5.0
    yield "ratio12_192k", signals.kind_clip("speechlike", 0.3, 192000), 192000, 40.0, 250.0, 7.3


def main():
    ref = oracle.reference()
    if ref is None:
        raise SystemExit("build oracle/_ref first (make -C oracle)")
    index = {"generator": "reference WORLD Harvest via oracle/_ref", "cases": []}
    for name, x, fs, lo, hi, period in cases():
        x = np.ascontiguousarray(x, dtype=np.float64)
        f0, t = ref.harvest(x, fs, lo, hi, period)
        fname = name + ".npz"
        np.savez_compressed(os.path.join(HERE, fname), x=x, f0=f0, times=t)
        index["cases"].append(dict(file=fname, fs=fs, f0_floor=lo, f0_ceil=hi, frame_period=period,
                                   samples=int(x.size), voiced=int((f0 > 0).sum())))
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1)
    print(json.dumps(index, indent=1))


if __name__ == "__main__":
    main()
