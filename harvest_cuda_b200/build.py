"""Builds the engine's shared library, ``libharvest_b200.so``, in this
directory from ``csrc/`` with nvcc for sm_100a (B200).

``--fmad=false`` and ``-ffp-contract=off`` keep separately rounded multiplies
and adds wherever the source writes them, as the reference's build does
(its CMakeLists.txt:40-46); kernels that want fused multiply-adds call
``fma()`` explicitly.

Usage: ``python -m harvest_cuda_b200.build [--force] [--verbose]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD_DIR = os.path.join(HERE, "_build")
LIBRARY = os.path.join(HERE, "libharvest_b200.so")
PEAKS_LIBRARY = os.path.join(HERE, "libhv_peaks.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["decimate.cu", "bandbank.cu", "bandbank_fft.cu", "candidates.cu", "refine.cu", "contour.cu",
           "metrics.cu", "bank_adjoint.cu", "engine.cu"]
HEADERS = ["hv_device.cuh", "hv_stages.cuh", "hv_events.cuh", "fft4096.cuh", "hv_runtime.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler",
                "-fPIC,-ffp-contract=off,-fvisibility=hidden", "-I" + INCLUDE]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build the engine")
    return path


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, ptxas_info=False):
    """Compile every CUDA source and link the library; returns its path."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS]
    headers.append(os.path.join(INCLUDE, "harvest_b200.h"))
    objects, jobs = [], []
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD_DIR, src.replace(".cu", ".o"))
        objects.append(obj)
        if force or ptxas_info or _stale(obj, [path] + headers):
            jobs.append([nvcc(), *FLAGS, *extra, "-c", path, "-o", obj])

    def run(cmd):
        out = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, out

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        for cmd, out in pool.map(run, jobs):
            if verbose or ptxas_info:
                sys.stdout.write(out.stdout + out.stderr)
            if out.returncode != 0:
                raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + out.stdout + out.stderr)
    if force or jobs or _stale(LIBRARY, objects):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIBRARY, *objects]
        out = subprocess.run(cmd, capture_output=True, text=True)
        if out.returncode != 0:
            raise RuntimeError("link failed:\n" + " ".join(cmd) + "\n" + out.stdout + out.stderr)
    # Measurement aid used by bench.py only (FP64 FMA peak).
    peaks_src = os.path.join(CSRC, "peaks.cu")
    if force or _stale(PEAKS_LIBRARY, [peaks_src]):
        cmd = [nvcc(), *FLAGS, "-shared", peaks_src, "-o", PEAKS_LIBRARY]
        out = subprocess.run(cmd, capture_output=True, text=True)
        if out.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + out.stdout + out.stderr)
    return LIBRARY


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers/spills per kernel")
    args = ap.parse_args()
    print(build(args.force, args.verbose, args.ptxas_info))


if __name__ == "__main__":
    main()
