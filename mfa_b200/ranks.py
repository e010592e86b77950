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


def shard_by_weight(items: Sequence[T], weights: Sequence[float], rank: int, world: int) -> list:
    """Whole systems for one rank, balanced by weight (bead count): greedy
    longest-processing-time assignment -- systems in decreasing weight, each to
    the rank with the least weight so far (ties to the lower rank, equal
    weights in index order), so every rank computes the same partition with no
    communication.  A rank's systems keep their original order; with one rank
    it is the whole list."""
    if len(items) != len(weights):
        raise ValueError("one weight per item")
    order = sorted(range(len(items)), key=lambda k: (-float(weights[k]), k))
    load = [0.0] * world
    owner = [0] * len(items)
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[k] = r
        load[r] += float(weights[k])
    return [items[k] for k in range(len(items)) if owner[k] == rank]


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
