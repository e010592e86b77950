"""The multi-rank bookkeeping of bench.py on CPU: two gloo ranks on this host
(127.0.0.1) shard whole systems, agree on the job's time as the largest of
their own, and sum their bead counts, with the same collective steps in the
same order on both ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from mfa_b200.ranks import max_over_ranks, shard, shard_by_weight, sum_over_ranks


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
    mine_w = shard_by_weight(list(range(10)), [3, 9, 1, 7, 7, 2, 8, 5, 4, 6], rank, world)
    t = max_over_ranks(1.0 + rank, dist)            # each rank's own time
    n = sum_over_ranks(float(len(mine) * 100), dist)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, mine, t, n, mine_w))


def test_shard_covers_every_system_once():
    items = list(range(11))
    parts = [shard(items, r, 4) for r in range(4)]
    assert sorted(sum(parts, [])) == items
    assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1


def test_shard_by_weight_balances_bead_counts():
    # uneven systems in the bead-count range of the batch workload
    import numpy as np
    rng = np.random.default_rng(3)
    w = [int(x) for x in rng.integers(1_000, 40_000, size=64)]
    items = list(range(64))
    for world in (1, 2, 3, 4, 8):
        parts = [shard_by_weight(items, w, r, world) for r in range(world)]
        assert sorted(sum(parts, [])) == items                      # every system once
        assert all(p == sorted(p) for p in parts)                   # original order kept
        loads = [sum(w[k] for k in p) for p in parts]
        # greedy LPT: the largest load exceeds the mean by at most one system
        assert max(loads) <= sum(w) / world + max(w)
        rr = [sum(w[k] for k in shard(items, r, world)) for r in range(world)]
        assert max(loads) <= max(rr)
    assert shard_by_weight(items, w, 0, 1) == items
    # a skewed case where every-world-th dealing is poor
    w2 = [100, 1, 100, 1, 100, 1, 100, 1]
    parts = [shard_by_weight(list(range(8)), w2, r, 2) for r in range(2)]
    assert [sum(w2[k] for k in p) for p in parts] == [202, 202]


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
    (r0, m0, t0, n0, w0), (r1, m1, t1, n1, w1) = res
    assert m0 == [0, 2, 4, 6, 8] and m1 == [1, 3, 5, 7, 9]
    # each rank computed the bead-count partition on its own: complementary, balanced
    assert sorted(w0 + w1) == list(range(10)) and w0 == [1, 2, 4, 7, 8] and w1 == [0, 3, 5, 6, 9]
    assert t0 == t1 == 2.0                       # the slower rank's time for both
    assert n0 == n1 == 1000.0


def test_without_process_group():
    assert max_over_ranks(3.5) == 3.5 and sum_over_ranks(2.0) == 2.0


def _small_systems():
    from mfa_b200 import configs
    return [configs.melt(seed=60 + k, n_chain=4 + 2 * k, n_mon=8, density=0.7) for k in range(5)]


def _step_with_oracle(cfg, steps=20):
    """The CPU stand-in for one rank's GPU work: the oracle advances the system
    and reports the per-system scalars a batch run gathers at its end."""
    from oracle import Oracle
    o = Oracle(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass)
    o.init_forces()
    for _ in range(steps):
        o.md_step()
    s = o.scalars()
    return [s["e_total"], s["v_total"], s["t_fluid"], float(s["n_rebuilds"])]


def _gather_main(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    from conftest import ROOT
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from mfa_b200.ranks import gather_system_values
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    systems = _small_systems()
    ids = shard_by_weight(list(range(len(systems))), [c.n for c in systems], rank, world)
    rows = [_step_with_oracle(systems[k]) for k in ids]
    table = gather_system_values(rows, ids, len(systems), dist)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, ids, table.tolist()))


def test_two_gloo_ranks_step_their_shards_and_gather_per_system_values():
    """Each rank steps its bead-count share of a small uneven batch (CPU
    stand-in: the oracle) and the per-system scalars are gathered into one
    table on every rank; it equals the same systems stepped in one process."""
    import numpy as np
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, ids0, t0), (_, ids1, t1) = res
    assert sorted(ids0 + ids1) == list(range(5)) and ids0 and ids1
    serial = np.array([_step_with_oracle(c) for c in _small_systems()])
    assert np.array_equal(np.array(t0), np.array(t1))          # every rank holds the same table
    assert np.array_equal(np.array(t0), serial)                # and it is the serial result, bit for bit


def test_gather_without_process_group_and_ownership_check():
    from mfa_b200.ranks import gather_system_values
    t = gather_system_values([[1.0, 2.0], [3.0, 4.0]], [1, 0], 2)
    assert t.tolist() == [[3.0, 4.0], [1.0, 2.0]]
    with pytest.raises(RuntimeError):
        gather_system_values([[1.0]], [0], 2)                   # system 1 computed nowhere
