"""Replica parallelism host logic on CPU: world_size 2 over gloo (no GPU)."""
from __future__ import annotations

import os

import pytest
import torch.multiprocessing as mp

from rooftop_mom_b200.replicas import max_over_ranks, shard, sum_over_ranks


def test_shard_covers_every_item_once():
    items = list(range(23))
    parts = [shard(items, r, 4) for r in range(4)]
    assert sorted(sum(parts, [])) == items
    assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1
    with pytest.raises(ValueError):
        shard(items, 4, 4)


def _worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard(range(10), rank, world)
        t = 1.0 + rank                       # a rank-dependent elapsed time
        out[rank] = (len(mine), max_over_ranks(t), sum_over_ranks(len(mine)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_over_gloo():
    import random

    port = 29500 + random.randint(0, 2000)
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    assert out[0][1] == out[1][1] == 2.0       # max over ranks
    assert out[0][2] == out[1][2] == 10.0      # every item solved once
