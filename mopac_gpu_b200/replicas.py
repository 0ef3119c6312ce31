"""Replica runs on several GPUs: one process per GPU, no data-path
collective.  The SCF of one molecule does not shard (the reference's
"2-GPU" path is a host-staged row split, cuda_wrappers.cu:272-461, which this
library does not reproduce); many molecules shard by molecule.  These helpers
are the host side of that: a cost-balanced split of a molecule list over the
ranks, and the max-over-ranks of a timing (the job is as slow as its slowest
rank).  They work with any torch.distributed backend (nccl on GPUs, gloo on
CPUs for the tests).
"""
from __future__ import annotations

import numpy as np


def shard(costs, rank: int, world: int) -> list:
    """Indices of the items rank `rank` of `world` runs: largest cost first,
    each item to the rank with the least total so far (ties to the lower
    rank).  Deterministic, disjoint, and together complete."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = np.zeros(world)
    mine = []
    for i in order:
        r = int(np.argmin(load))
        load[r] += float(costs[i])
        if r == rank:
            mine.append(i)
    return sorted(mine)


def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """The maximum of `value` over all ranks (the value itself without a
    process group)."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
