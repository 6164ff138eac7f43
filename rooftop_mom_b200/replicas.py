"""Replica parallelism: independent plate solves spread over ranks, one process per GPU.

A single plate's solve does not shard (its FFTs and dot products are global), so N GPUs run N independent
replicas: every rank takes its share of the work items, no collective touches the data path, and the
elapsed time of the job is the maximum over ranks (device-timed by each rank).
"""
from __future__ import annotations


def shard(items, rank: int, world: int):
    """The items of `rank` (round robin, so uneven sizes spread over ranks)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("rank must lie in [0, world)")
    return list(items)[rank::world]


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over the ranks of the default process group (the value itself without one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
