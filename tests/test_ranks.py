"""The multi-rank bookkeeping of bench.py on CPU: two gloo ranks on this host
(127.0.0.1) shard whole systems, agree on the job's time as the largest of
their own, and sum their bead counts, with the same collective steps in the
same order on both ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from mfa_b200.ranks import max_over_ranks, shard, sum_over_ranks


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mine = shard(list(range(10)), rank, world)
    t = max_over_ranks(1.0 + rank, dist)            # each rank's own time
    n = sum_over_ranks(float(len(mine) * 100), dist)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, mine, t, n))


def test_shard_covers_every_system_once():
    items = list(range(11))
    parts = [shard(items, r, 4) for r in range(4)]
    assert sorted(sum(parts, [])) == items
    assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1


def test_two_gloo_ranks_agree_on_time_and_size():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, t0, n0), (r1, m1, t1, n1) = res
    assert m0 == [0, 2, 4, 6, 8] and m1 == [1, 3, 5, 7, 9]
    assert t0 == t1 == 2.0                       # the slower rank's time for both
    assert n0 == n1 == 1000.0


def test_without_process_group():
    assert max_over_ranks(3.5) == 3.5 and sum_over_ranks(2.0) == 2.0
