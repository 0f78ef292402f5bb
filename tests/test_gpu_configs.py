"""The engine at the full sizes of the benchmark workloads that the 16 kHz
batch does not reach, against the CPU checker (the reference's bundled WORLD
build when present), clip by clip, at the acceptance bar (time axis
bit-exact, voicing agreement on >= 99.9 % of frames, every jointly voiced
frame within 1e-6 relative):

* 64 clips of U(2, 30) s at 48 kHz, base F0 U(60, 600) Hz, SNR U(0, 20) dB,
  71-800 Hz, 1 ms frames: decimation ratio 6, WORLD's direct branch for a
  1 ms period (harvest.cpp:1230-1235), clips up to 1.44 M samples and 30,001
  frames, through the batched graph path;
* one 60 s clip at 44.1 kHz (voiced vibrato segments alternating with pink
  noise, 30 dB SNR), 71-800 Hz, 5 ms frames: 2.6 M samples and 60,001
  analysis frames, through both the plain per-clip call and the batch path.

The checker runs one clip per spawned worker process on the host cores."""
import numpy as np
import pytest

import harvest_cuda_b200 as hv
import oracle
from harvest_cuda_b200 import signals
from tests.test_gpu_parity import assert_parity

pytestmark = pytest.mark.gpu


def test_batch64_48k_full_size(gpu):
    wl = signals.workload("batch64_48k", seed=1000)
    clips, fs = wl["clips"], wl["fs"]
    settings = (wl["f0_floor"], wl["f0_ceil"], wl["frame_period"])
    assert len(clips) == 64 and fs == 48000 and settings == (71.0, 800.0, 1.0)
    longest = max(len(c) for c in clips)
    assert longest > 28 * fs        # the longest clip is close to the 30 s maximum
    ours = hv.harvest_many(clips, fs, *settings)
    expected = oracle.harvest_many(clips, fs, *settings)
    voiced = 0
    for i, (a, e) in enumerate(zip(ours, expected)):
        assert len(a[0]) == hv.output_length(len(clips[i]), fs, 1.0)
        m = assert_parity(a, e)
        voiced += m["joint_voiced_frames"]
    assert voiced > 100000


def test_clip60s_44k_full_size(gpu, checker):
    wl = signals.workload("clip60s_44k", seed=1000)
    x, fs = wl["clips"][0], wl["fs"]
    settings = (wl["f0_floor"], wl["f0_ceil"], wl["frame_period"])
    assert x.size == 60 * 44100
    expected = checker.harvest(x, fs, *settings)
    single = hv.harvest(x, fs, *settings)
    m = assert_parity(single, expected)
    assert m["joint_voiced_frames"] > 3000
    batched = hv.harvest_many([x], fs, *settings)[0]
    np.testing.assert_array_equal(batched[0], single[0])
    np.testing.assert_array_equal(batched[1], single[1])
