"""The multi-GPU host logic of bench.py on two gloo ranks (CPU): each rank
draws its own batch, the timing reduction takes the slowest rank, and the
whole-job rate counts every rank's prices.  Rendezvous on 127.0.0.1."""
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
        P, I = bench.make_batch(16, bench.rank_seed(0, rank))
        # ranks report different times; every rank sees the maximum
        t = bench.max_over_ranks(1.0 + rank, dist, world, "cpu")
        rate = bench.aggregate_rate(world, 16, 3, t)
        out[rank] = (float(P[:, 0].sum()), t, rate)
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_reduce():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    (s0, t0, r0), (s1, t1, r1) = out[0], out[1]
    assert s0 != s1                      # each rank priced its own contracts
    assert t0 == t1 == 2.0               # the slowest rank's time
    assert r0 == r1 == world * 16 * 3 / 2.0


def test_rank_batches_are_reproducible():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    a, _ = bench.make_batch(8, bench.rank_seed(3, 1))
    b, _ = bench.make_batch(8, bench.rank_seed(3, 1))
    assert np.array_equal(a, b)
