"""Clip sharding across ranks (one process per GPU).

Clips are independent, so a batch splits across ranks with no data-path
exchange: each rank runs Harvest on its share on its own GPU, and one
all-gather of the ragged outputs (host objects, once per call) returns the
whole batch to every rank. Shares are balanced by longest-processing-time
on clip length, the dominant cost of every stage.
"""
from __future__ import annotations

import heapq

import numpy as np

__all__ = ["partition", "harvest_sharded"]


def partition(lengths, world):
    """Longest-processing-time assignment of clips to `world` ranks.
    Returns one sorted list of clip indices per rank."""
    if world < 1:
        raise ValueError("world must be positive")
    heap = [(0, r) for r in range(world)]
    shares = [[] for _ in range(world)]
    for i in sorted(range(len(lengths)), key=lambda i: (-int(lengths[i]), i)):
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + int(lengths[i]), r))
    return [sorted(s) for s in shares]


def harvest_sharded(clips, fs, f0_floor=71.0, f0_ceil=800.0, frame_period=5.0, *, group=None,
                    compute=None):
    """Harvest on a list of clips split across the ranks of `group` (the
    default torch.distributed group). Every rank passes the same clip list
    and receives every clip's ``(f0, times)`` in order. ``compute(clips)``
    returns the local results; by default it is ``harvest_many`` on this
    rank's current CUDA device."""
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    shares = partition([len(c) for c in clips], world)
    mine = shares[rank]
    if compute is None:
        import torch

        from .api import harvest_many
        device = torch.cuda.current_device()

        def compute(local):
            return harvest_many(local, fs, f0_floor, f0_ceil, frame_period, device=device)
    local = compute([clips[i] for i in mine]) if mine else []
    gathered = [None] * world
    dist.all_gather_object(gathered, [(i, np.asarray(f), np.asarray(t)) for i, (f, t) in zip(mine, local)],
                           group=group)
    out = [None] * len(clips)
    for part in gathered:
        for i, f, t in part:
            out[i] = (f, t)
    return out
