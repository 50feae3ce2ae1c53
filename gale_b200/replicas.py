"""Multi-GPU layout of this path: independent problems, one process per GPU.

The Stokes problems of a batch (or the replicas of one benchmark problem) are independent,
so they shard across ranks with no data-path collective: rank r takes problems
r, r + world, r + 2·world, …  Only the timing needs the process group: a barrier around
the timed region and the maximum of the per-rank device times.  Slab decomposition of a
single large problem (face-halo exchange + FP64 allreduce of the Krylov dots) is not
part of this package.
"""
from __future__ import annotations

from typing import List, Sequence


def shard(items: Sequence, rank: int, world: int) -> List:
    """Round-robin share of `items` for `rank` (every item on exactly one rank)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    return [items[i] for i in range(rank, len(items), world)]


def max_over_ranks(value: float, group=None, device=None) -> float:
    """Maximum of a per-rank scalar (step time) over the process group."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sum_over_ranks(value: float, group=None, device=None) -> float:
    """Sum of a per-rank count (problems solved) over the process group."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())
