"""The multi-rank clip sharding path on CPU: world size 2 over gloo, with the
C restatement of Harvest standing in for each rank's GPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from harvest_cuda_b200.distributed import partition
from harvest_cuda_b200 import signals


def test_partition_is_balanced_and_complete():
    rng = np.random.default_rng(0)
    lengths = rng.integers(16000, 192000, 256)
    for world in (1, 2, 3, 8):
        shares = partition(lengths, world)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(lengths)))
        loads = [int(lengths[s].sum()) for s in shares]
        assert max(loads) - min(loads) <= int(lengths.max())
    assert partition([5, 3], 4)[2:] == [[], []]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, result_path):
    import torch.distributed as dist

    import oracle
    from harvest_cuda_b200.distributed import harvest_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    clips = [signals.kind_clip(k, s, 16000) for k, s in
             [("speechlike", 0.3), ("high", 0.25), ("low", 0.4), ("silence", 0.1), ("speechlike", 0.2)]]
    calls = []

    def compute(local):
        calls.append(len(local))
        return [oracle.port().harvest(x, 16000) for x in local]

    out = harvest_sharded(clips, 16000, compute=compute)
    ok = all(np.array_equal(out[i][0], oracle.port().harvest(clips[i], 16000)[0]) and
             np.array_equal(out[i][1], oracle.port().harvest(clips[i], 16000)[1]) for i in range(len(clips)))
    with open(f"{result_path}.{rank}", "w") as f:
        f.write(f"{int(ok)} {calls[0] if calls else 0}")
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_results_match_single_process(tmp_path):
    world = 2
    path = str(tmp_path / "result")
    mp.start_processes(_worker, args=(world, _free_port(), path), nprocs=world, start_method="spawn")
    got = [open(f"{path}.{r}").read().split() for r in range(world)]
    assert all(ok == "1" for ok, _ in got)
    assert sum(int(n) for _, n in got) == 5        # every clip computed exactly once
    assert all(int(n) > 0 for _, n in got)         # both ranks worked
