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


def gather_system_values(values, index, n_total: int, dist=None, device="cpu"):
    """The per-system values of every rank in one table: rank r holds rows
    `values` (m_r x k) of the systems with global indices `index` (m_r); every
    rank gets the n_total x k table, with one collective (a sum of disjoint
    rows -- as an all-gather of the shards, without padding uneven shards).
    A count column checks that every system was computed on exactly one rank.
    Without a process group the local rows are the table."""
    import numpy as np
    vals = np.asarray(values, dtype=np.float64).reshape(len(index), -1)
    k = vals.shape[1] if vals.size else 0
    if dist is not None:
        import torch
        kk = torch.tensor([float(k)], dtype=torch.float64, device=device)
        dist.all_reduce(kk, op=dist.ReduceOp.MAX)
        k = int(kk.item())
    table = np.zeros((n_total, k + 1))
    for row, g in zip(vals, index):
        table[g, :k] = row
        table[g, k] += 1.0
    if dist is not None:
        import torch
        t = torch.from_numpy(table).to(device)
        dist.all_reduce(t)
        table = t.cpu().numpy()
    if not (table[:, k] == 1.0).all():
        raise RuntimeError("a system was computed on no rank or on several")
    return table[:, :k]
