"""Throughput benchmark of the Harvest engine (one JSON line on rank 0).

Workload (default): the ragged batch of 256 clips at 16 kHz, lengths
uniform 1-12 s (about 1.7k audio seconds), floor 50 Hz, ceil 1100 Hz,
frame_period 5 ms; synthetic seeded glide clips (F0 100 -> 250 Hz, 10
harmonics, 20 dB SNR, 0.3 s unvoiced noise at both ends). A step is one
pass of the whole Harvest pipeline over that batch.

* ``value``: audio seconds per second with the batch resident in HBM,
  through the C ABI with device pointers (one replayed CUDA graph per step),
  timed with CUDA events on the launching stream; max over ranks.
* ``e2e``: the same metric through the public host-memory API: per step,
  the host-to-device copy of the step's input from pinned memory, compute,
  and the device-to-host copy of f0 and times, with ``BatchPipeline``
  overlapping each step's copies with its neighbours' compute;
  ``e2e.blocking`` is ``harvest_batch`` doing the three in turn.
* ``per_clip``: the plain per-clip path (``harvest`` once per clip).
* ``roofline``: the band bank (the largest stage): its algorithmic FP64
  FLOP rate (WORLD's FFT model) over its CUDA-event duration (stage-timed
  steps) against the FP64 FMA throughput measured on the same GPU, the
  stage's binding bound; beside it the stage-boundary byte rate against the
  measured HBM copy bandwidth.
* ``cpu_baseline``: the reference's bundled WORLD Harvest (oracle/_ref) on
  the host cores over a bounded sample of the same batch (median of 3).
* ``configs``: the other workloads (one 3 s clip at 16 kHz, one 60 s clip
  at 44.1 kHz, 64 clips of 2-30 s at 48 kHz with 1 ms frames), each timed
  the same way; single clips add the per-call latency of ``harvest()`` and
  WORLD on one host core.
* ``grad``: the F0 gradient (``harvest_cuda_b200.autograd``) on 32 clips of
  4 s at 16 kHz from the same generator, L = sum over voiced frames of
  (f0 - true f0)^2: forward + backward device milliseconds per audio second
  (CUDA events), and the agreement of dL/dx with central finite differences
  (eps 1e-6) at 64 random samples per clip.

``--impl reference`` times that CPU implementation alone on every host core
over every clip of the workload (the K timed steps together make one pass;
median of three passes) and prints the same line with
``"impl": "reference"``. It never loads the engine's library: the workload
generator is loaded by path, not through the package.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (fs, floor, ceil, period, description)
    "batch256_16k": "256 clips x U(1,12) s at 16 kHz, floor 50, ceil 1100, period 5 ms",
    "batch64_48k": "64 clips x U(2,30) s at 48 kHz, floor 71, ceil 800, period 1 ms",
    "clip60s_44k": "1 clip of 60 s at 44.1 kHz, floor 71, ceil 800, period 5 ms",
    "clip3s_16k": "1 clip of 3 s at 16 kHz, floor 71, ceil 800, period 5 ms",
    "grad32x4s_16k": "F0 gradient only: 32 clips x 4 s at 16 kHz, floor 71, ceil 800, period 5 ms",
}


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="batch256_16k")
    ap.add_argument("--cpu-seconds", type=float, default=8.0,
                    help="target duration of one pass of the CPU baseline sample (3 passes)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip timing the other workloads (one 3 s clip, one 60 s clip, 64 clips at 48 kHz)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-per-clip", action="store_true")
    ap.add_argument("--no-grad", action="store_true", help="skip the F0-gradient measurement")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="with --impl reference: skip timing the reference's own CUDA path")
    ap.add_argument("--grad-fd-samples", type=int, default=64,
                    help="random samples per clip for the finite-difference check (0: none)")
    ap.add_argument("--clips", type=int, default=0,
                    help="use only the first N clips of the workload (small profiling runs)")
    return ap.parse_args()


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------- models --
LN2 = 0.69314718055994529


def clip_params(n, fs, floor, ceil):
    """Per-clip analysis sizes (reference src/engine.cpp:255-266)."""
    ratio = min(12, max(1, int(fs / 8000.0 + 0.5)))
    fs_r = fs / ratio
    lo, hi = floor * 0.9, ceil * 1.1
    bands = 1 + int(math.log(hi / lo) / LN2 * 40.0)
    y_len = -(-n // ratio)
    first = lo * 2.0 ** (1 / 40.0)
    m = y_len + 5 + 2 * int(2.0 * fs_r / first)
    nfft = int(2.0 ** (int(math.log(m) / LN2) + 1.0))
    frames = int(1000.0 * n / fs) + 1
    return dict(ratio=ratio, bands=bands, y_len=y_len, nfft=nfft, frames=frames,
                capacity=7 * int(bands / 10.0 + 0.5))


def band_bank_models(lengths, fs, floor, ceil):
    """Algorithmic bytes and FP64 FLOPs of the band-pass bank stage for a
    batch: per clip, the filtered band signals written and read once
    (16 B x bands x y_len) plus the per-band candidates (16 B x bands x
    frames); FLOPs of one n-point real inverse FFT and spectrum product per
    band, 2.5 n log2 n + 6 (n/2 + 1), with the filter spectra cached."""
    nbytes = flops = 0.0
    for n in lengths:
        p = clip_params(int(n), fs, floor, ceil)
        nbytes += 16.0 * p["bands"] * p["y_len"] + 16.0 * p["bands"] * p["frames"]
        nf = p["nfft"]
        flops += p["bands"] * (2.5 * nf * math.log2(nf) + 6.0 * (nf / 2 + 1))
    return nbytes, flops


def byte_model(lengths, fs, floor, ceil, period):
    """Stage-boundary byte model of the whole pipeline per batch."""
    total = 0.0
    for n in lengths:
        p = clip_params(int(n), fs, floor, ceil)
        out = int(1000.0 * n / fs / period) + 1
        total += (8.0 * n + 16.0 * p["y_len"] + 16.0 * p["bands"] * p["y_len"]
                  + 16.0 * p["bands"] * p["frames"] + 32.0 * p["frames"] * p["capacity"]
                  + 16.0 * out)
    return total


# ------------------------------------------------------------- workloads --
def signals_module():
    """``harvest_cuda_b200/signals.py`` loaded by its path. The generators
    need only NumPy; importing them through the package would run its
    ``__init__``, which loads the engine's shared library, and the reference
    arm must not map that library."""
    import importlib.util
    name = "hv_bench_signals"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(
            name, os.path.join(ROOT, "harvest_cuda_b200", "signals.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def make_workload(name, seed, clips=0):
    signals = signals_module()
    wl = signals.workload(name, seed=seed)
    if clips:
        wl["clips"] = wl["clips"][:clips]
    packed, offsets = signals.pack(wl["clips"])
    return dict(packed=packed, offsets=offsets, fs=wl["fs"], floor=wl["f0_floor"],
                ceil=wl["f0_ceil"], period=wl["frame_period"],
                lengths=np.diff(offsets).tolist())


# --------------------------------------------------------------- clocks --
CLOCK_QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


class ClockSampler:
    """Samples the SM clock and the clock-event reasons while the timed
    region runs: through NVML every 10 ms (read-only queries, in a thread;
    the first sample is taken before the region starts), else nvidia-smi
    every 200 ms."""

    REASONS = (("hw_slowdown", "HwSlowdown"), ("hw_thermal_slowdown", "HwThermalSlowdown"),
               ("sw_thermal_slowdown", "SwThermalSlowdown"), ("sw_power_cap", "SwPowerCap"))

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.thread = None
        self.samples = []       # (sm MHz, max sm MHz, set of reasons)
        self.source = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.device)
        bus = f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}.0"
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def _nvml_sample(self, nv, h, mx):
        mask = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        reasons = {name for name, suffix in self.REASONS
                   if mask & getattr(nv, "nvmlClocksEventReason" + suffix)}
        self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), mx, reasons))

    def __enter__(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._nvml_sample(nv, h, mx)
        except Exception:           # no NVML binding or device: fall back to nvidia-smi
            nv = None
        if nv is not None:
            self._nv = nv
            self.source = "nvml, 10 ms"
            self._stop = threading.Event()

            def loop():
                while not self._stop.wait(0.01):
                    try:
                        self._nvml_sample(nv, h, mx)
                    except Exception:
                        return
            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            return self
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={CLOCK_QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi, 200 ms"
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self._stop.set()
            self.thread.join(timeout=5)
            try:
                self._nv.nvmlShutdown()   # balances the nvmlInit of __enter__
            except Exception:
                pass
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            for ln in out.splitlines():
                parts = [p.strip() for p in ln.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm, mx = float(parts[1]), float(parts[2])
                except ValueError:
                    continue
                reasons = {name for (name, _), flag in zip(self.REASONS, parts[5:9])
                           if flag.lower() == "active"}
                self.samples.append((sm, mx, reasons))

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        reasons = set().union(*(r for _, _, r in self.samples))
        return {"sm_mhz": statistics.median(sm for sm, _, _ in self.samples),
                "sm_max_mhz": self.samples[-1][1], "reasons": sorted(reasons),
                "samples": len(self.samples), "source": self.source}


# ------------------------------------------------------- CPU baseline --
def _world_clip(args):
    x, fs, floor, ceil, period = args
    import oracle
    checker = oracle.best()
    t0 = time.perf_counter()
    f0, _ = checker.harvest(x, fs, floor, ceil, period)
    return time.perf_counter() - t0, checker.name, f0


def cpu_sample(wl, target_seconds, cores):
    """Clips of the workload whose CPU time is about target_seconds on
    `cores` cores, at about 2.5 audio-s/s per core (floor 50 Hz, 190 bands)."""
    budget = target_seconds * cores * 2.5 * wl["fs"]
    chosen, total = [], 0
    offs = wl["offsets"]
    for i in range(len(offs) - 1):
        n = int(offs[i + 1] - offs[i])
        if total + n > budget and chosen:
            break
        chosen.append(i)
        total += n
    return chosen


def run_cpu(pool, wl, clips, repeats=1):
    """WORLD on `clips` of the workload, one clip per worker process, the
    longest submitted first so that no core idles behind a long clip at the
    end. Returns (audio seconds, median wall seconds over `repeats` passes,
    checker kind, every pass's wall seconds)."""
    offs, x = wl["offsets"], wl["packed"]
    order = sorted(clips, key=lambda i: offs[i] - offs[i + 1])
    tasks = [(np.ascontiguousarray(x[offs[i]:offs[i + 1]]), wl["fs"], wl["floor"], wl["ceil"],
              wl["period"]) for i in order]
    walls = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        results = pool.map(_world_clip, tasks, chunksize=1)
        walls.append(time.perf_counter() - t0)
    audio = sum(t[0].size for t in tasks) / wl["fs"]
    kind = "reference" if results and results[0][1] == "reference" else "port"
    by_clip = dict(zip(order, (r[2] for r in results)))
    run_cpu.last_f0 = [by_clip[i] for i in clips]
    return audio, statistics.median(walls), kind, walls


def cpu_model():
    """The host CPU's model name (from /proc/cpuinfo)."""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def mapped_libraries():
    """Shared objects mapped into this process (from /proc/self/maps)."""
    try:
        with open("/proc/self/maps") as f:
            return sorted({ln.split()[-1] for ln in f if ln.rstrip().endswith(".so") or ".so." in ln})
    except OSError:
        return []


def accuracy_against(reference_f0, sample, f0, out_off, kind, device):
    """The engine's batch output (the last end-to-end step) against the CPU
    reference's F0 for the sampled clips, compared per clip on the device
    (metrics.compare_batch) and summarised over the sample."""
    from harvest_cuda_b200.metrics import compare_batch
    ours = np.concatenate([f0[out_off[i]:out_off[i + 1]] for i in sample])
    ref = np.concatenate(reference_f0)
    offsets = np.concatenate([[0], np.cumsum([len(r) for r in reference_f0])])
    stats = compare_batch(ref, ours, offsets, device=device)
    frames = sum(s["frames"] for s in stats)
    both = (ref > 0) & (ours > 0)
    rel = np.abs(ours[both] - ref[both]) / ref[both]
    p99 = [s["cents_p99"] for s in stats if s["cents_p99"] is not None]
    cmax = [s["cents_max"] for s in stats if s["cents_max"] is not None]
    return {"against": "WORLD Harvest (oracle/_ref)" if kind == "reference" else "C restatement (oracle)",
            "clips": len(stats), "frames": frames,
            "vuv_disagreement": sum(s["vuv_disagreement"] * s["frames"] for s in stats) / max(frames, 1),
            "cents_p99_max_over_clips": max(p99) if p99 else None, "cents_max": max(cmax) if cmax else None,
            "over_600_cents": sum(s["over_600_cents"] for s in stats),
            "voiced_f0_rel_max": float(rel.max()) if rel.size else None,
            "computed_on": "device, hv_compare_batch (rel_max on the host)"}


def kernels_per_step(ratio):
    # finiteness flag; decimation (3 kernels per direction, or one copy at
    # ratio 1); DC removal and edge bins (chunk sums, removal, bins); block
    # spectra and the FFT band bank; official candidates; refinement (keys,
    # two bucket passes, offsets, jobs); prune + best; contour (prepare,
    # extend, finish).
    return 1 + (6 if ratio > 1 else 1) + 3 + 2 + 1 + 5 + 1 + 3


def fp64_peak(device):
    import ctypes as ct
    path = os.path.join(ROOT, "harvest_cuda_b200", "libhv_peaks.so")
    if not os.path.exists(path):
        return None
    lib = ct.CDLL(path)
    out = ct.c_double(0.0)
    if lib.hv_peak_fp64(int(device), ct.byref(out)) != 0:
        return None
    return out.value


# ------------------------------------------------------ reference arm --
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.workload == "grad32x4s_16k":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no F0 gradient"}), flush=True)
        return
    cores = os.cpu_count() or 1
    world = int(os.environ.get("WORLD_SIZE", "1"))
    wl = make_workload(args.workload, seed=1000, clips=args.clips)
    offs = wl["offsets"]
    every = list(range(len(offs) - 1))
    pool = mp.get_context("spawn").Pool(cores)
    # Warm-up steps: one of the shortest clips per worker (starts the
    # workers and loads the library in each).
    shortest = sorted(every, key=lambda i: offs[i + 1] - offs[i])[:cores]
    for _ in range(args.warmup):
        run_cpu(pool, wl, shortest)
    # Timed: the K steps together are one pass over every clip of the
    # workload (step k is the k-th K-th of the batch); the pass runs through
    # one worker pool, longest clip first, so that no core idles at a step
    # boundary. The pass is repeated three times and the median is reported.
    repeats = 3
    audio, wall, kind, walls = run_cpu(pool, wl, every, repeats=repeats)
    pool.close()
    pool.join()
    value = audio / wall
    maps = mapped_libraries()
    engine_maps = [m for m in maps if "libharvest_b200" in m]
    if engine_maps:
        raise RuntimeError(f"the reference arm mapped the engine's library: {engine_maps}")
    base = {"value": value, "unit": "audio-s/s", "cores": cores, "cpu_model": cpu_model(),
            "kind": kind, "repeats": repeats, "pass_walls_s": [round(w, 3) for w in walls],
            "sample": f"every clip of the workload ({len(every)} clips, {audio:.1f} audio-s) per pass, "
                      f"split over the {args.steps} timed steps, one clip per worker process "
                      f"(WORLD is single-threaded), longest first; median of {repeats} passes"}
    line = {
        "impl": "reference", "metric": "batched audio-s/s (16 kHz)", "value": value,
        "unit": "audio-s/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * wall / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, wl, world),
        "cpu_baseline": base,
        "e2e": {"value": value, "unit": "audio-s/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if not args.no_reference_cuda:
        line["reference_cuda"] = reference_cuda_measure(wl)
    line["libraries_mapped"] = [m for m in mapped_libraries() if ROOT in m]
    print(json.dumps(line), flush=True)


def reference_cuda_measure(wl, budget_s=60.0):
    """The reference's own GPU path (oracle/_ref/libref_cuda.so, its
    src/cuda_backend.cu + src/engine.cpp) on the workload's clips, one clip per
    call as its API takes them, host arrays in and out; wall clock over
    consecutive clips until all are done or `budget_s` has passed."""
    import oracle
    ref = oracle.reference_cuda()
    if ref is None:
        return {"unavailable": "oracle/_ref/libref_cuda.so was not built"}
    if not ref.available(0):
        return {"unavailable": "the reference's CUDA build does not run on device 0"}
    offs, x = wl["offsets"], wl["packed"]
    clips = [np.ascontiguousarray(x[offs[i]:offs[i + 1]]) for i in range(len(offs) - 1)]
    for c in clips[:3]:
        ref.harvest(c, wl["fs"], wl["floor"], wl["ceil"], wl["period"])
    done = audio = 0
    t0 = time.perf_counter()
    for c in clips:
        ref.harvest(c, wl["fs"], wl["floor"], wl["ceil"], wl["period"])
        done += 1
        audio += len(c) / wl["fs"]
        if time.perf_counter() - t0 > budget_s:
            break
    wall = time.perf_counter() - t0
    return {"value": audio / wall, "unit": "audio-s/s", "clips": done, "audio_seconds": audio,
            "wall_s": wall, "path": "reference src/cuda_backend.cu + src/engine.cpp analyze(), "
                                    "per clip, host buffers, built for sm_100a by oracle/Makefile"}


# ------------------------------------------------------------ our arm --
def run_grad_only(args):
    """--workload grad32x4s_16k: the F0-gradient measurement as the line."""
    import torch
    import harvest_cuda_b200 as hv
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    g = grad_measure(hv, args.steps, max(3, args.warmup), stream, fd_per_clip=args.grad_fd_samples)
    line = {"metric": g.pop("metric"), "value": g.pop("value"), "unit": g.pop("unit"), "n_gpus": 1,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": g["fwd_ms"] + g["bwd_ms"],
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": args.workload, "description": WORKLOADS[args.workload]},
            "grad": g}
    print(json.dumps(line), flush=True)


def run_ours(args):
    if args.workload == "grad32x4s_16k":
        run_grad_only(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cores = os.cpu_count() or 1
    # The CPU pool starts before any GPU call (spawned workers).
    pool = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        pool = mp.get_context("spawn").Pool(cores)
    wl = make_workload(args.workload, seed=1000 + rank, clips=args.clips)

    import datetime
    import ctypes as ct
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    import harvest_cuda_b200 as hv
    from harvest_cuda_b200 import _native

    fs, floor, ceil, period = wl["fs"], wl["floor"], wl["ceil"], wl["period"]
    offsets = np.ascontiguousarray(wl["offsets"], dtype=np.int64)
    clips = offsets.size - 1
    audio = float(offsets[-1]) / fs
    out_off = hv.api._out_offsets(offsets, fs, period)
    x_dev = torch.from_numpy(wl["packed"]).to(f"cuda:{local}")
    f0_dev = torch.empty(int(out_off[-1]), dtype=torch.float64, device=f"cuda:{local}")
    t_dev = torch.empty_like(f0_dev)
    # A dedicated stream: torch's default is the legacy NULL stream, which the
    # C ABI maps to the engine's own stream.
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    off_ptr = offsets.ctypes.data_as(ct.POINTER(ct.c_int64))

    def device_step(flags=0):
        status = _native.lib.hv_harvest_batch(
            x_dev.data_ptr(), off_ptr, clips, fs, floor, ceil, period, local, f0_dev.data_ptr(),
            t_dev.data_ptr(), _native.HV_DEVICE_POINTERS | flags, stream.cuda_stream)
        _native.raise_for(status)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # --- value: device-resident batch, replayed graph, CUDA events. The first
    # warm-up call autotunes the refinement launch shape for this batch.
    for _ in range(max(3, args.warmup)):
        device_step()
    torch.cuda.synchronize()
    tuning = (ct.c_int * 3)()
    _native.raise_for(_native.lib.hv_last_tuning(tuning))
    barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            device_step()
        end.record(stream)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ms = max_over_ranks(start.elapsed_time(end) / args.steps)
    value = audio * world / (ms / 1000.0)

    # --- stage-timed steps: per-stage CUDA events on the same stream.
    stage_steps = max(3, min(args.steps, 5))
    acc = np.zeros(_native.HV_STAGE_COUNT)
    buf = np.zeros(_native.HV_STAGE_COUNT)
    for _ in range(stage_steps):
        device_step(_native.HV_RECORD_STAGES)
        _native.raise_for(_native.lib.hv_last_stage_ms(buf.ctypes.data_as(ct.POINTER(ct.c_double))))
        acc += buf
    stage_ms = acc / stage_steps
    names = [_native.lib.hv_stage_name(i).decode() for i in range(_native.HV_STAGE_COUNT)]
    stages = dict(zip(names, stage_ms.round(4).tolist()))

    # --- e2e: public API from pinned host memory. Each step uploads its
    # batch and downloads its f0 and times. BatchPipeline overlaps those
    # copies with the neighbouring steps' compute; harvest_batch (blocking)
    # runs them in turn and is reported beside it.
    from harvest_cuda_b200.pipeline import BatchPipeline
    pinned = torch.from_numpy(wl["packed"]).pin_memory()
    x_host = pinned.numpy()
    pipe = BatchPipeline(fs, floor, ceil, period, device=local, depth=2)
    for _ in range(pipe.depth):          # every slot's buffers allocated before timing
        pipe.submit(x_host, offsets)
    while pipe.pending():
        pipe.result()
    barrier()
    laps = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        pipe.submit(x_host, offsets)
        if pipe.pending() == pipe.depth:
            f0, times, _ = pipe.result()
            laps.append(time.perf_counter())
    while pipe.pending():
        f0, times, _ = pipe.result()
        laps.append(time.perf_counter())
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps)
    barrier()
    laps = np.diff(np.concatenate([[t0], laps])) * 1000.0
    e2e = {"value": audio * world / e2e_s, "unit": "audio-s/s",
           "h2d_bytes_per_step": int(x_host.nbytes), "d2h_bytes_per_step": int(f0.nbytes + times.nbytes),
           "ms_per_step": e2e_s * 1000.0, "ms_median": float(np.median(laps)),
           "api": "harvest_cuda_b200.pipeline.BatchPipeline (depth 2): copies overlapped across steps"}
    hv.harvest_batch(x_host, offsets, fs, floor, ceil, period, device=local)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        f0, times, _ = hv.harvest_batch(x_host, offsets, fs, floor, ceil, period, device=local)
    blocking_s = max_over_ranks((time.perf_counter() - t0) / args.steps)
    barrier()
    e2e["blocking"] = {"value": audio * world / blocking_s, "ms_per_step": blocking_s * 1000.0,
                       "api": "harvest_cuda_b200.harvest_batch: upload, compute, download in turn"}

    line = None
    if rank == 0:
        line = summarize(args, wl, value, ms, stages, e2e, clocks.summary(), local, world)
        line["autotuned"] = {"refine_min_blocks_per_sm": tuning[0], "refine_grid_blocks_per_sm": tuning[1],
                             "key": "fs, f0 range, log2 of the batch's samples, log2 of its longest clip's frames"}
        if world == 1 and not args.no_per_clip:
            line["per_clip"] = per_clip(hv, wl, local)
            line["batched_over_per_clip"] = round(e2e["value"] / line["per_clip"]["value"], 2)
        if world == 1 and not args.no_grad:
            line["grad"] = grad_measure(hv, args.steps, max(3, args.warmup), stream,
                                        fd_per_clip=args.grad_fd_samples)
        if world == 1 and not args.no_configs:
            line["configs"] = {name: config_measure(hv, name, local, args.steps, args.warmup, stream, pool)
                               for name in EXTRA_CONFIGS if name != args.workload}
        if pool is not None:
            sample = cpu_sample(wl, args.cpu_seconds, cores)
            a, wall, kind, walls = run_cpu(pool, wl, sample, repeats=3)
            pool.close()
            line["cpu_baseline"] = {
                "value": a / wall, "unit": "audio-s/s", "cores": cores, "cpu_model": cpu_model(),
                "kind": kind, "repeats": 3, "pass_walls_s": [round(w, 3) for w in walls],
                "sample": f"{len(sample)} of the batch's clips ({a:.1f} audio-s), one clip per "
                          f"worker process, longest first; median of 3 passes, {wall:.1f} s wall"}
            line["accuracy"] = accuracy_against(run_cpu.last_f0, sample, f0, out_off, kind, local)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def stage_models(wl):
    """Algorithmic bytes (and FP64 FLOPs where a model exists) per stage for
    one pass over the batch, from the stage-boundary byte model."""
    fs, floor, ceil, period = wl["fs"], wl["floor"], wl["ceil"], wl["period"]
    models = {k: [0.0, None] for k in
              ("decimate", "band_bank", "candidates", "refine", "prune", "contour")}
    for n in wl["lengths"]:
        p = clip_params(int(n), fs, floor, ceil)
        fr, cap, bands = p["frames"], p["capacity"], p["bands"]
        out = int(1000.0 * n / fs / period) + 1
        models["decimate"][0] += 8.0 * n + 16.0 * p["y_len"]
        models["candidates"][0] += 8.0 * bands * fr + 8.0 * fr * cap / 7
        models["refine"][0] += 8.0 * fr * cap / 7 + 32.0 * fr * cap
        models["prune"][0] += 64.0 * fr * cap
        models["contour"][0] += 32.0 * fr * cap + 16.0 * out
    nbytes, flops = band_bank_models(wl["lengths"], fs, floor, ceil)
    models["band_bank"] = [nbytes, flops]
    return models


def ncu_traffic(stage, wl):
    """DRAM bytes per launch of `stage` for this workload, scaled by audio
    seconds from the ncu capture summarised in profiles/ (None if absent)."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        per = json.load(f)["bytes_per_audio_second"].get(stage)
    return None if per is None else per * float(sum(wl["lengths"])) / wl["fs"]


def workload_config(args, wl, world):
    """The `config` object of the JSON line, shared by both arms so that
    they describe the same workload the same way."""
    return {"workload": args.workload, "description": WORKLOADS[args.workload],
            "clips_per_gpu": len(wl["lengths"]),
            "audio_seconds_per_gpu": float(sum(wl["lengths"])) / wl["fs"],
            "l2": "inputs and working set larger than L2 (no flush)",
            "parallelism": f"clip sharding, {world} GPU(s), no collective"}


def roofline(wl, stages, device, traffic=True):
    """The band bank's roofline: its algorithmic FP64 FLOP rate (WORLD's FFT
    model) against the FP64 FMA throughput measured on this GPU, which is
    the binding bound of the stage, and beside it the stage-boundary byte
    rate against the measured HBM copy bandwidth."""
    hbm, hbm_src = load_peaks()
    nbytes, flops = stage_models(wl)["band_bank"]
    dur = stages["band_bank"] / 1000.0
    peak64 = fp64_peak(device)
    hbm_part = {"hbm_achieved_gbs": nbytes / dur / 1e9, "hbm_peak_gbs": hbm,
                "hbm_frac": nbytes / dur / 1e9 / hbm, "hbm_peak_source": hbm_src,
                "algorithmic_bytes": nbytes}
    common = {"kernel": "band_bank", "dominant_stage": max(stages, key=stages.get),
              "launch_ms": stages["band_bank"],
              "traffic": ncu_traffic("band_bank", wl) if traffic else None}
    if peak64:
        return {"bound": "fp64", "achieved": flops / dur / 1e12, "peak": peak64, "unit": "TFLOP/s",
                "frac": flops / dur / 1e12 / peak64, "algorithmic_flops": flops,
                "peak_source": "measured: FP64 FMA loop on this GPU (libhv_peaks)", **common, **hbm_part}
    return {"bound": "hbm", "achieved": hbm_part["hbm_achieved_gbs"], "peak": hbm, "unit": "GB/s",
            "frac": hbm_part["hbm_frac"], "peak_source": hbm_src, **common, **hbm_part}


def summarize(args, wl, value, ms, stages, e2e, clocks, device, world):
    roof = roofline(wl, stages, device)
    ratio = clip_params(int(wl["lengths"][0]), wl["fs"], wl["floor"], wl["ceil"])["ratio"]
    return {
        "metric": "batched audio-s/s (16 kHz)", "value": value, "unit": "audio-s/s",
        "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(args, wl, world),
        "stage_ms": stages, "roofline": roof, "e2e": e2e, "clocks": clocks,
        "gpu_launches": kernels_per_step(ratio) * args.steps,
        "model_bytes_per_step": byte_model(wl["lengths"], wl["fs"], wl["floor"], wl["ceil"],
                                           wl["period"]),
    }


def grad_measure(hv, steps, warmup, stream, fd_per_clip=64, eps=1e-6):
    """F0-gradient forward + backward time per audio second on 32 x 4 s
    clips at 16 kHz, and dL/dx against central finite differences of the
    GPU forward pass."""
    import torch
    from harvest_cuda_b200 import autograd, signals
    w = signals.workload("grad32x4s_16k", seed=7)
    fs, floor, ceil, period = w["fs"], w["f0_floor"], w["f0_ceil"], w["frame_period"]
    clips, truths = w["clips"], w["truths"]
    offsets = tuple(int(v) for v in np.concatenate([[0], np.cumsum([len(c) for c in clips])]))
    audio = offsets[-1] / fs
    x = torch.from_numpy(np.concatenate(clips)).cuda()
    counts = [hv.output_length(len(c), fs, period) for c in clips]
    times = np.concatenate([np.arange(n) * period / 1000.0 for n in counts])
    target_np = np.concatenate([tr(t) for tr, t in zip(truths, np.split(times, np.cumsum(counts)[:-1]))])
    target = torch.from_numpy(target_np).cuda()

    def step():
        xs = x.detach().requires_grad_(True)
        f0, _ = autograd.HarvestF0.apply(xs, offsets, fs, floor, ceil, period)
        voiced = (f0.detach() > 0) & (target > 0)
        loss = ((f0 - target) ** 2 * voiced).sum()
        return xs, f0, loss

    for _ in range(warmup):
        xs, f0, loss = step()
        loss.backward()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    fwd = bwd = 0.0
    for _ in range(steps):
        ev[0].record(stream)
        xs, f0, loss = step()
        ev[1].record(stream)
        loss.backward()
        ev[2].record(stream)
        torch.cuda.synchronize()
        fwd += ev[0].elapsed_time(ev[1])
        bwd += ev[1].elapsed_time(ev[2])
    fwd, bwd = fwd / steps, bwd / steps
    # Finite differences of the forward pass at random samples.
    grad = xs.grad.cpu().numpy()
    f0n = f0.detach().cpu().numpy()
    rng = np.random.default_rng(0)
    g, fd, scale, switched, flipped = [], [], [], 0, 0
    o = np.concatenate([[0], np.cumsum(counts)])
    for c, clip in enumerate(clips if fd_per_clip > 0 else []):
        base_f0, tgt = f0n[o[c]:o[c + 1]], target_np[o[c]:o[c + 1]]
        voiced = (base_f0 > 0) & (tgt > 0)
        positions = rng.choice(len(clip), fd_per_clip, replace=False)
        batch = []
        for p in positions:
            for s in (eps, -eps):
                xp = clip.copy()
                xp[p] += s
                batch.append(xp)
        out = hv.harvest_many(batch, fs, floor, ceil, period)
        for k, p in enumerate(positions):
            up, down = out[2 * k][0], out[2 * k + 1][0]
            if not (np.array_equal(up > 0, base_f0 > 0) and np.array_equal(down > 0, base_f0 > 0)):
                flipped += 1
                continue
            # L differences frame by frame: (a - t)^2 - (b - t)^2 = (a - b)(a + b - 2t).
            central = np.sum(((up - down) * (up + down - 2 * tgt))[voiced]) / (2 * eps)
            curvature = np.sum(((up - base_f0) * (up + base_f0 - 2 * tgt) -
                                (base_f0 - down) * (base_f0 + down - 2 * tgt))[voiced]) / eps
            if abs(curvature) > 1e-3 * max(abs(central), 1.0):
                switched += 1
                continue
            g.append(grad[offsets[c] + p])
            fd.append(central)
            scale.append(np.abs(grad[offsets[c]:offsets[c + 1]]).max())
    g, fd, scale = np.array(g), np.array(fd), np.array(scale)
    fd_report = None
    if g.size:
        fd_report = {
            "eps": eps, "samples": int(g.size), "voicing_flips": flipped, "candidate_switches": switched,
            "rel_error_norm": float(np.linalg.norm(g - fd) / np.linalg.norm(fd)),
            "rel_error_max": float(np.max(np.abs(g - fd) / scale)),
            "rel_error_note": "norm-wise over the samples; max is per sample |g - fd| over the "
                              "clip's max |dL/dx| (difference noise at eps 1e-6 is ~1e-6 absolute)"}
    return {
        "metric": "F0-grad fwd+bwd ms/s", "value": (fwd + bwd) / audio, "unit": "ms per audio-s",
        "higher_is_better": False, "fwd_ms": fwd, "bwd_ms": bwd, "steps": steps,
        "workload": "32 clips x 4 s at 16 kHz (glide generator), floor 71, ceil 800, period 5 ms",
        "audio_seconds": audio,
        "finite_differences": fd_report,
    }


EXTRA_CONFIGS = ("clip3s_16k", "clip60s_44k", "batch64_48k")


def config_measure(hv, name, device, steps, warmup, stream, pool):
    """Another workload of the benchmark set, timed as the headline one:
    device-resident steps through the C ABI (graph replay, CUDA events),
    stage times, end to end from pinned host memory through BatchPipeline,
    and the band bank's roofline. A single clip adds the per-call latency of
    harvest() (host arrays in and out), and, with a worker pool, the
    reference's WORLD on one host core (three single-threaded runs in
    parallel processes, median) with the engine's agreement with it."""
    import ctypes as ct
    import torch
    from harvest_cuda_b200 import _native
    from harvest_cuda_b200.pipeline import BatchPipeline
    wl = make_workload(name, seed=1000)
    fs, floor, ceil, period = wl["fs"], wl["floor"], wl["ceil"], wl["period"]
    offsets = np.ascontiguousarray(wl["offsets"], dtype=np.int64)
    clips = offsets.size - 1
    audio = float(offsets[-1]) / fs
    out_off = hv.api._out_offsets(offsets, fs, period)
    dev = torch.device("cuda", device)
    x_dev = torch.from_numpy(wl["packed"]).to(dev)
    f0_dev = torch.empty(int(out_off[-1]), dtype=torch.float64, device=dev)
    t_dev = torch.empty_like(f0_dev)
    off_ptr = offsets.ctypes.data_as(ct.POINTER(ct.c_int64))

    def step(flags=0):
        _native.raise_for(_native.lib.hv_harvest_batch(
            x_dev.data_ptr(), off_ptr, clips, fs, floor, ceil, period, device, f0_dev.data_ptr(),
            t_dev.data_ptr(), _native.HV_DEVICE_POINTERS | flags, stream.cuda_stream))

    for _ in range(max(3, warmup)):
        step()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        step()
    end.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(end) / steps
    acc = np.zeros(_native.HV_STAGE_COUNT)
    buf = np.zeros(_native.HV_STAGE_COUNT)
    for _ in range(3):
        step(_native.HV_RECORD_STAGES)
        _native.raise_for(_native.lib.hv_last_stage_ms(buf.ctypes.data_as(ct.POINTER(ct.c_double))))
        acc += buf
    names = [_native.lib.hv_stage_name(i).decode() for i in range(_native.HV_STAGE_COUNT)]
    stages = dict(zip(names, (acc / 3).round(4).tolist()))
    pinned = torch.from_numpy(wl["packed"]).pin_memory()
    x_host = pinned.numpy()
    pipe = BatchPipeline(fs, floor, ceil, period, device=device, depth=2)
    for _ in range(pipe.depth):
        pipe.submit(x_host, offsets)
    while pipe.pending():
        pipe.result()
    t0 = time.perf_counter()
    for _ in range(steps):
        pipe.submit(x_host, offsets)
        if pipe.pending() == pipe.depth:
            f0, times, _ = pipe.result()
    while pipe.pending():
        f0, times, _ = pipe.result()
    e2e_s = (time.perf_counter() - t0) / steps
    out = {"description": WORKLOADS[name], "clips": clips, "audio_seconds": audio,
           "device_ms_per_step": ms, "value": audio / (ms / 1000.0), "unit": "audio-s/s",
           "stage_ms": stages,
           "e2e": {"value": audio / e2e_s, "unit": "audio-s/s", "ms_per_step": e2e_s * 1000.0,
                   "h2d_bytes_per_step": int(x_host.nbytes),
                   "d2h_bytes_per_step": int(f0.nbytes + times.nbytes),
                   "api": "harvest_cuda_b200.pipeline.BatchPipeline (depth 2)"},
           "roofline": roofline(wl, stages, device, traffic=False)}
    if clips == 1:
        x = np.ascontiguousarray(wl["packed"])
        for _ in range(3):
            hv.harvest(x, fs, floor, ceil, period, device=device)
        laps = []
        for _ in range(max(steps, 5)):
            t0 = time.perf_counter()
            f0, times = hv.harvest(x, fs, floor, ceil, period, device=device)
            laps.append(time.perf_counter() - t0)
        out["latency_ms"] = {"median": 1000.0 * statistics.median(laps), "min": 1000.0 * min(laps),
                             "calls": len(laps),
                             "api": "harvest_cuda_b200.harvest (NumPy in and out, one call per clip)"}
        if pool is not None:
            task = (x, fs, floor, ceil, period)
            results = pool.map(_world_clip, [task] * 3, chunksize=1)
            wall = statistics.median(r[0] for r in results)
            ref = results[0][2]
            both = (ref > 0) & (f0 > 0)
            rel = np.abs(f0[both] - ref[both]) / ref[both]
            out["cpu_single_thread"] = {
                "value": audio / wall, "unit": "audio-s/s", "seconds_per_clip": wall, "cores": 1,
                "cpu_model": cpu_model(), "kind": results[0][1], "repeats": 3,
                "sample": "the whole clip; three single-threaded runs in parallel worker processes, median"}
            out["accuracy"] = {"against": "WORLD Harvest (oracle/_ref)" if results[0][1] == "reference"
                               else "C restatement (oracle)",
                               "frames": int(ref.size),
                               "vuv_disagreement": float(np.mean((ref > 0) != (f0 > 0))),
                               "voiced_f0_rel_max": float(rel.max()) if rel.size else None}
    return out


def per_clip(hv, wl, device):
    """The plain per-clip path: harvest() once per clip, host buffers."""
    offs, x = wl["offsets"], wl["packed"]
    clips = [np.ascontiguousarray(x[offs[i]:offs[i + 1]]) for i in range(len(offs) - 1)]
    for c in clips[:4]:
        hv.harvest(c, wl["fs"], wl["floor"], wl["ceil"], wl["period"], device=device)
    t0 = time.perf_counter()
    for c in clips:
        hv.harvest(c, wl["fs"], wl["floor"], wl["ceil"], wl["period"], device=device)
    wall = time.perf_counter() - t0
    audio = float(offs[-1]) / wl["fs"]
    return {"value": audio / wall, "unit": "audio-s/s", "ms_per_pass": 1000.0 * wall}


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
