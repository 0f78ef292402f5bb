"""Batches from host memory with the copies overlapped: while the GPU runs
Harvest on one batch, the next batch's samples travel host -> device and the
previous batch's F0 travels back.

``harvest_batch`` (the NumPy API) does upload, compute and download in
turn, so every call pays its own PCIe transfers on top of the compute (on
the 256-clip 16 kHz batch: 209 MB up, 5 MB down, about 5 ms of a 49 ms
call). A stream of batches (a corpus being analysed, a serving queue) can
hide them: ``BatchPipeline.submit`` enqueues a batch and returns without
waiting for the GPU, ``result`` returns the oldest outstanding batch's
``(f0, times, out_offsets)``. Results equal ``harvest_batch``'s bit for bit.

    pipe = BatchPipeline(16000, 50.0, 1100.0, 5.0)
    for packed, offsets in batches:
        pipe.submit(packed, offsets)
        if pipe.pending() == pipe.depth:
            f0, times, out_offsets = pipe.result()
    while pipe.pending():
        f0, times, out_offsets = pipe.result()

Three CUDA streams per pipeline: uploads, compute (the engine's device-
pointer entry point), downloads; ``depth`` slots of device and pinned host
buffers rotate between batches, each reuse ordered behind the slot's
previous download by CUDA events. Inputs already in page-locked memory (for
example ``torch.empty(n, dtype=torch.float64).pin_memory().numpy()``) are
uploaded directly; other arrays are first copied into the slot's pinned
staging buffer on the host. A batch with a non-finite sample raises
``ValueError`` from ``result`` (the check runs on the device and comes back
with the F0, so ``submit`` never waits for it; the engine is given zeros in
place of such samples).
"""
from __future__ import annotations

import collections
import ctypes as ct

import numpy as np
import torch

from . import _native
from .api import _as_float, _as_int, _check_array, _out_offsets

__all__ = ["BatchPipeline"]


class _Slot:
    def __init__(self, device):
        self.device = device
        self.x = None          # device samples
        self.f0 = None         # device outputs
        self.times = None
        self.ok = torch.zeros((), dtype=torch.bool, device=device)
        self.staging = None    # pinned host input copy (unpinned inputs only)
        self.host_f0 = None    # pinned host outputs
        self.host_times = None
        self.host_ok = torch.zeros((), dtype=torch.bool).pin_memory()
        self.uploaded = torch.cuda.Event()
        self.computed = torch.cuda.Event()
        self.downloaded = torch.cuda.Event()

    def buffers(self, n_in, n_out):
        if self.x is None or self.x.numel() < n_in:
            self.x = torch.empty(n_in, dtype=torch.float64, device=self.device)
        if self.f0 is None or self.f0.numel() < n_out:
            self.f0 = torch.empty(n_out, dtype=torch.float64, device=self.device)
            self.times = torch.empty(n_out, dtype=torch.float64, device=self.device)
            self.host_f0 = torch.empty(n_out, dtype=torch.float64).pin_memory()
            self.host_times = torch.empty(n_out, dtype=torch.float64).pin_memory()


class BatchPipeline:
    """Harvest on a stream of host batches with uploads, compute and
    downloads overlapped across consecutive batches.

    ``fs``, ``f0_floor``, ``f0_ceil``, ``frame_period`` and ``device`` are
    those of ``harvest_batch``; ``depth`` (>= 2) is the number of batches in
    flight."""

    def __init__(self, fs, f0_floor=71.0, f0_ceil=800.0, frame_period=5.0, *, device=0, depth=2,
                 graph=True):
        self.fs = _as_int(fs, "fs")
        self.f0_floor = _as_float(f0_floor, "f0_floor")
        self.f0_ceil = _as_float(f0_ceil, "f0_ceil")
        self.frame_period = _as_float(frame_period, "frame_period")
        self.device_index = _as_int(device, "device")
        self.depth = _as_int(depth, "depth")
        if self.depth < 2:
            raise ValueError("depth must be at least 2")
        if not torch.cuda.is_available():
            raise RuntimeError("BatchPipeline needs a CUDA device")
        self.flags = _native.HV_DEVICE_POINTERS | (0 if graph else _native.HV_NO_GRAPH)
        dev = torch.device("cuda", self.device_index)
        self._dev = dev
        self._up = torch.cuda.Stream(dev)
        self._run = torch.cuda.Stream(dev)
        self._down = torch.cuda.Stream(dev)
        self._slots = [_Slot(dev) for _ in range(self.depth)]
        self._next = 0
        self._queue = collections.deque()   # (slot, out_offsets, clips' output count)

    def pending(self):
        """Batches submitted and not yet returned by ``result``."""
        return len(self._queue)

    def submit(self, x, offsets):
        """Enqueue one batch (``x``, ``offsets`` as for ``harvest_batch``)
        and return without waiting for the GPU. Raises ``RuntimeError`` when
        ``depth`` batches are already outstanding (call ``result`` first)."""
        if len(self._queue) == self.depth:
            raise RuntimeError("all pipeline slots are in use; call result() first")
        x = _check_array(x)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        if offsets.ndim != 1 or offsets.size < 2:
            raise ValueError("offsets must hold clips + 1 entries")
        if offsets[0] < 0 or offsets[-1] > x.size or np.any(np.diff(offsets) < 0):
            raise ValueError("offsets must be nondecreasing and lie within x")
        if np.any(np.diff(offsets) <= 0):
            raise ValueError(f"clip {int(np.argmax(np.diff(offsets) <= 0))} is empty")
        out_off = _out_offsets(offsets, self.fs, self.frame_period)
        lo, hi = int(offsets[0]), int(offsets[-1])
        n_in, n_out = hi - lo, int(out_off[-1])
        local = offsets - lo

        slot = self._slots[self._next]
        self._next = (self._next + 1) % self.depth
        # The slot's previous batch was returned by result(), so its download
        # (and with it its compute and upload) has completed.
        slot.buffers(n_in, n_out)
        part = x[lo:hi]
        src = torch.from_numpy(part) if part.flags.writeable else None
        if src is None or not src.is_pinned():
            if slot.staging is None or slot.staging.numel() < n_in:
                slot.staging = torch.empty(n_in, dtype=torch.float64).pin_memory()
            np.copyto(slot.staging[:n_in].numpy(), part)
            src = slot.staging[:n_in]
        with torch.cuda.stream(self._up):
            slot.x[:n_in].copy_(src, non_blocking=True)
            slot.uploaded.record(self._up)
        self._run.wait_event(slot.uploaded)
        with torch.cuda.stream(self._run):
            xs = slot.x[:n_in]
            torch.all(torch.isfinite(xs), out=slot.ok)
            # A batch with a non-finite sample is rejected at result(); the
            # engine is given zeros in its place.
            torch.nan_to_num_(xs, nan=0.0, posinf=0.0, neginf=0.0)
            status = _native.lib.hv_harvest_batch(
                xs.data_ptr(), local.ctypes.data_as(ct.POINTER(ct.c_int64)), local.size - 1, self.fs,
                self.f0_floor, self.f0_ceil, self.frame_period, self.device_index, slot.f0.data_ptr(),
                slot.times.data_ptr(), self.flags, ct.c_void_p(self._run.cuda_stream))
            _native.raise_for(status)
            slot.computed.record(self._run)
        self._down.wait_event(slot.computed)
        with torch.cuda.stream(self._down):
            slot.host_f0[:n_out].copy_(slot.f0[:n_out], non_blocking=True)
            slot.host_times[:n_out].copy_(slot.times[:n_out], non_blocking=True)
            slot.host_ok.copy_(slot.ok, non_blocking=True)
            slot.downloaded.record(self._down)
        # Device buffers are used on other streams than the one they were
        # allocated on; keep the caching allocator from reusing them early.
        for t in (slot.x, slot.f0, slot.times, slot.ok):
            t.record_stream(self._up)
            t.record_stream(self._run)
            t.record_stream(self._down)
        self._queue.append((slot, out_off, n_out))

    def result(self):
        """``(f0, times, out_offsets)`` of the oldest outstanding batch, as
        NumPy arrays owned by the caller; waits for its download."""
        if not self._queue:
            raise RuntimeError("no batch outstanding")
        slot, out_off, n_out = self._queue.popleft()
        slot.downloaded.synchronize()
        if not bool(slot.host_ok):
            raise ValueError("x must contain only finite samples")
        return slot.host_f0[:n_out].numpy().copy(), slot.host_times[:n_out].numpy().copy(), out_off
