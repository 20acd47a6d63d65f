"""Batched cases sharded across ranks: two gloo ranks on the CPU agree on a
disjoint, complete and balanced assignment without exchanging it."""
import os

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from canard_b200 import shard
from canard_b200.cases import batched


def _worker(rank, world, port, sizes, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = shard.my_cases(sizes, world, rank)
    t = torch.zeros(len(sizes), dtype=torch.int64)
    t[mine] = rank + 1
    dist.all_reduce(t)  # each case claimed exactly once: sum of (rank+1) over owners
    load = torch.tensor([sum(sizes[i] for i in mine)], dtype=torch.int64)
    loads = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(loads, load)
    if rank == 0:
        out.put((t.tolist(), [int(x.item()) for x in loads], mine))
    dist.barrier()
    dist.destroy_process_group()


def test_assign_is_a_partition():
    sizes = [c.npts for c in batched(16, lo=32, hi=40)]
    for world in (1, 2, 3, 8):
        parts = shard.assign(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)
    with pytest.raises(ValueError):
        shard.assign(sizes, 0)


def test_two_gloo_ranks_agree():
    sizes = [c.npts for c in batched(12, lo=32, hi=44)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    claims, loads, mine0 = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    # every case owned by exactly one rank: claims are 1 (rank 0) or 2 (rank 1)
    assert all(c in (1, 2) for c in claims)
    assert sum(loads) == sum(sizes)
    assert mine0 == shard.my_cases(sizes, 2, 0)
