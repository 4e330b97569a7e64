"""The multi-GPU host logic on two gloo ranks (CPU): one batch is split across
ranks by estimated solve cost, each rank prices its shard, one all-gather
returns the whole price vector to every rank, the timing reduction takes the
slowest rank and the whole-job rate counts every rank's prices.  The pricing
function here is the CPU oracle (these tests have no GPU); the GPU path runs
the same sharding with the engine.  Rendezvous on 127.0.0.1."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # ranks report different times; every rank sees the maximum
        t = bench.max_over_ranks(1.0 + rank, dist, world, "cpu")
        rate = bench.aggregate_rate(world, 16, 3, t)
        from fpe_option_b200 import sharding

        P, I = _small_batch()
        p, st = sharding.price_sharded(P, I, _oracle_prices, dist, "cpu", rank, world)
        mine = sharding.partition(sharding.solve_costs(P, I), world)[rank]
        out[rank] = (t, rate, p.tolist(), st.tolist(), mine.tolist())
    finally:
        dist.destroy_process_group()


def _small_batch():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    P, I = bench.make_batch(8, 5)
    I[:, 0] = np.where(np.arange(8) % 3 == 0, 16, 12)  # small grids: the oracle prices them in seconds
    I[:, 1] = np.where(np.arange(8) % 2 == 0, 10, 8)
    P[1, 9], I[1, 2] = 85.0, 0  # a down-and-in call: two solves, twice the cost
    return P, I


def _oracle_prices(P, I):
    from oracle import pyoracle as po

    opt = po.options(disc=1, rtol=1e-4, atol=1e-6, complex_direct=1, radau_constants=2)
    return po.price_batch(P, I, opt), np.zeros(len(P), np.int32)


def test_two_ranks_shard_gather_and_reduce():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    (t0, r0, p0, s0, m0), (t1, r1, p1, s1, m1) = out[0], out[1]
    assert t0 == t1 == 2.0               # the slowest rank's time
    assert r0 == r1 == world * 16 * 3 / 2.0
    assert m0 and m1 and not set(m0) & set(m1)  # disjoint non-empty shards
    assert sorted(m0 + m1) == list(range(8))
    # every rank holds the whole vector, bit for bit the 1-rank prices
    P, I = _small_batch()
    ref, _ = _oracle_prices(P, I)
    assert p0 == p1 == ref.tolist()
    assert s0 == s1 == [0] * 8


def test_partition_balances_cost():
    from fpe_option_b200 import sharding

    rng = np.random.default_rng(0)
    c = rng.uniform(1.0, 10.0, 257)
    for world in (1, 2, 4, 8):
        shards = sharding.partition(c, world)
        assert sorted(np.concatenate(shards).tolist()) == list(range(257))
        loads = np.array([c[s].sum() for s in shards])
        assert loads.max() - loads.min() <= c.max()  # LPT: within one job of even
        again = sharding.partition(c, world)
        assert all(np.array_equal(a, b) for a, b in zip(shards, again))


def test_costs_count_knock_ins_twice():
    from fpe_option_b200 import sharding

    P = np.zeros((2, 12))
    P[:, 5] = 1.0
    I = np.array([[32, 16, 8], [32, 16, 0]], np.int32)
    c = sharding.solve_costs(P, I)
    assert c[1] == 2 * c[0]
