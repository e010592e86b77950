"""Rank bookkeeping of multi-GPU runs (one process per GPU).

A single system is not decomposed (the reference has no decomposition and a
system fits one GPU many times over): N GPUs run N independent replicas, or
share out whole independent systems.  Nothing but timing crosses ranks: every
rank times its own work on its own stream, and the job's time is the largest
of them (all ranks take the same collective steps in the same order)."""
from __future__ import annotations

import os
from typing import Sequence, TypeVar

T = TypeVar("T")


def rank_env():
    """(world size, rank, local rank) as torch.distributed.run exports them."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(items: Sequence[T], rank: int, world: int) -> list:
    """Whole systems for one rank: every world-th one, starting at `rank`."""
    return list(items[rank::world])


def max_over_ranks(x: float, dist=None, device="cpu") -> float:
    """The largest value of x over the ranks (x itself without a process group)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, dist=None, device="cpu") -> float:
    """The sum of x over the ranks (x itself without a process group)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t)
    return float(t.item())
