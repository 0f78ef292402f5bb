"""TEST INFRASTRUCTURE ONLY: ctypes front end for the two CPU checkers.

* ``port()``: the C restatement in ``harvest_oracle.c`` (``liboracle.so``).
* ``reference()``: the reference's own bundled WORLD Harvest compiled from the
  reference sources by ``Makefile`` into ``_ref/libworld_ref.so``; ``None``
  when that library was never built.
* ``reference_cuda()``: the reference's own CUDA path (its
  ``src/cuda_backend.cu`` + ``src/engine.cpp``) compiled by ``Makefile`` into
  ``_ref/libref_cuda.so``; ``None`` when absent. It runs on the GPU and serves
  as a second parity reference and the timed reference GPU path.

Only tests, ``__graft_entry__.smoke()`` and the reference legs of ``bench.py``
(its CPU baseline and ``--impl reference``) import this package, and only as
the checker or the timed reference. The engine under ``harvest_cuda_b200``
never does.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libworld_ref.so")
REF_CUDA_LIB = os.path.join(HERE, "_ref", "libref_cuda.so")

_D = ct.POINTER(ct.c_double)
_I = ct.POINTER(ct.c_int)


def build(quiet=True):
    """Compile both checkers (the reference one only where its tree exists)."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _ptr(a, kind=_D):
    return a.ctypes.data_as(kind)


class Checker:
    """One CPU implementation of Harvest with stage dumps."""

    def __init__(self, path, name):
        self.name = name
        self.lib = ct.CDLL(path)
        lib = self.lib
        lib.oracle_params.argtypes = [ct.c_int, ct.c_int, ct.c_double, ct.c_double, _I]
        lib.oracle_output_length.argtypes = [ct.c_int, ct.c_int, ct.c_double]
        lib.oracle_output_length.restype = ct.c_int
        lib.oracle_harvest.argtypes = [_D, ct.c_int, ct.c_int, ct.c_double, ct.c_double,
                                       ct.c_double, _D, _D]
        lib.oracle_stages.argtypes = [_D, ct.c_int, ct.c_int, ct.c_double, ct.c_double,
                                      _D, _D, _I, _D, _D, _D, _D, _D, _D, _D, _D]
        lib.oracle_fix_contour.argtypes = [_D, _D, ct.c_int, ct.c_int, ct.c_int, _D]
        lib.oracle_fix_contour_base.argtypes = [_D, _D, _D, ct.c_int, ct.c_int, ct.c_int, _D]
        lib.oracle_smooth_contour.argtypes = [_D, ct.c_int, _D]

    def params(self, n, fs, f0_floor=71.0, f0_ceil=800.0):
        out = np.zeros(6, dtype=np.int32)
        self.lib.oracle_params(int(n), int(fs), float(f0_floor), float(f0_ceil), _ptr(out, _I))
        keys = ("ratio", "y_len", "fft_size", "bands", "frames", "capacity")
        return {k: int(v) for k, v in zip(keys, out)}

    def harvest(self, x, fs, f0_floor=71.0, f0_ceil=800.0, frame_period=5.0):
        x = np.ascontiguousarray(x, dtype=np.float64)
        m = self.lib.oracle_output_length(len(x), int(fs), float(frame_period))
        f0 = np.zeros(m)
        t = np.zeros(m)
        self.lib.oracle_harvest(_ptr(x), len(x), int(fs), float(f0_floor), float(f0_ceil),
                                float(frame_period), _ptr(t), _ptr(f0))
        return f0, t

    def stages(self, x, fs, f0_floor=71.0, f0_ceil=800.0):
        x = np.ascontiguousarray(x, dtype=np.float64)
        p = self.params(len(x), fs, f0_floor, f0_ceil)
        fr, cap = p["frames"], p["capacity"]
        out = dict(
            y=np.zeros(p["y_len"]), raw=np.zeros((p["bands"], fr)),
            cand=np.zeros((fr, cap)), refined=np.zeros((fr, cap)), scores=np.zeros((fr, cap)),
            pruned=np.zeros((fr, cap)), pruned_scores=np.zeros((fr, cap)),
            base=np.zeros(fr), fixed=np.zeros(fr), smoothed=np.zeros(fr))
        count = np.zeros(1, dtype=np.int32)
        self.lib.oracle_stages(
            _ptr(x), len(x), int(fs), float(f0_floor), float(f0_ceil), _ptr(out["y"]),
            _ptr(out["raw"]), _ptr(count, _I), _ptr(out["cand"]), _ptr(out["refined"]),
            _ptr(out["scores"]), _ptr(out["pruned"]), _ptr(out["pruned_scores"]),
            _ptr(out["base"]), _ptr(out["fixed"]), _ptr(out["smoothed"]))
        out["count"] = int(count[0])
        out["params"] = p
        return out

    def fix_contour(self, cand, scores, columns=None, base=None):
        """FixF0Contour on [frames][stride] candidate and score matrices
        (the first `columns` columns); with `base`, FixStep1-4 start from it
        instead of SearchF0Base's contour."""
        cand = np.ascontiguousarray(cand, dtype=np.float64)
        scores = np.ascontiguousarray(scores, dtype=np.float64)
        frames, stride = cand.shape
        if stride == 0:     # no candidate columns: keep the row pointers valid
            cand, scores, stride = np.zeros((frames, 1)), np.zeros((frames, 1)), 1
            columns = 0
        out = np.zeros(frames)
        cols = stride if columns is None else int(columns)
        if base is None:
            self.lib.oracle_fix_contour(_ptr(cand), _ptr(scores), frames, cols, stride, _ptr(out))
        else:
            base = np.ascontiguousarray(base, dtype=np.float64)
            self.lib.oracle_fix_contour_base(_ptr(base), _ptr(cand), _ptr(scores), frames, cols, stride,
                                             _ptr(out))
        return out

    def smooth_contour(self, f0):
        f0 = np.ascontiguousarray(f0, dtype=np.float64)
        out = np.zeros(len(f0))
        self.lib.oracle_smooth_contour(_ptr(f0), len(f0), _ptr(out))
        return out


_cache = {}


def port():
    if "port" not in _cache:
        if not os.path.exists(PORT_LIB):
            build()
        _cache["port"] = Checker(PORT_LIB, "port")
    return _cache["port"]


def reference():
    if "ref" not in _cache:
        _cache["ref"] = Checker(REF_LIB, "reference") if os.path.exists(REF_LIB) else None
    return _cache["ref"]


def best():
    """The reference build when present, else the restatement."""
    return reference() or port()


def _harvest_task(args):
    x, fs, f0_floor, f0_ceil, frame_period = args
    return best().harvest(x, fs, f0_floor, f0_ceil, frame_period)


def harvest_many(clips, fs, f0_floor=71.0, f0_ceil=800.0, frame_period=5.0, processes=None):
    """``best().harvest`` on every clip, one clip per worker process (WORLD
    is single-threaded), longest clip first. The workers are spawned, not
    forked, so this is safe in a process that has already used CUDA.
    Returns ``(f0, times)`` pairs in clip order."""
    import multiprocessing as mp
    order = sorted(range(len(clips)), key=lambda i: -len(clips[i]))
    tasks = [(np.ascontiguousarray(clips[i], dtype=np.float64), int(fs), float(f0_floor),
              float(f0_ceil), float(frame_period)) for i in order]
    workers = max(1, min(len(tasks), processes or os.cpu_count() or 1))
    with mp.get_context("spawn").Pool(workers) as pool:
        results = pool.map(_harvest_task, tasks, chunksize=1)
    out = [None] * len(clips)
    for i, r in zip(order, results):
        out[i] = r
    return out


class ReferenceCuda:
    """The reference's own GPU Harvest (one clip per call, as its API)."""

    def __init__(self, path):
        self.lib = ct.CDLL(path)
        self.lib.refcuda_last_error.restype = ct.c_char_p
        self.lib.refcuda_available.argtypes = [ct.c_int]
        self.lib.refcuda_harvest.argtypes = [_D, ct.c_int, ct.c_int, ct.c_double, ct.c_double,
                                             ct.c_double, ct.c_int, _D, _D, ct.c_int]

    def available(self, device=0):
        return bool(self.lib.refcuda_available(int(device)))

    def harvest(self, x, fs, f0_floor=71.0, f0_ceil=800.0, frame_period=5.0, device=0):
        x = np.ascontiguousarray(x, dtype=np.float64)
        m = int(1000.0 * len(x) / fs / frame_period) + 1
        f0, t = np.zeros(m), np.zeros(m)
        rc = self.lib.refcuda_harvest(_ptr(x), len(x), int(fs), float(f0_floor), float(f0_ceil),
                                      float(frame_period), int(device), _ptr(f0), _ptr(t), m)
        if rc != 0:
            raise RuntimeError(self.lib.refcuda_last_error().decode())
        return f0, t


def reference_cuda():
    if "ref_cuda" not in _cache:
        _cache["ref_cuda"] = ReferenceCuda(REF_CUDA_LIB) if os.path.exists(REF_CUDA_LIB) else None
    return _cache["ref_cuda"]
