"""One batch of contracts split across GPUs (one process per GPU).

Every solve is independent, so the batch shards with no exchange during the
solves: each rank prices the contracts assigned to it, and one all-gather of
the price and status vectors at the end gives every rank the whole batch in
its original order.  The assignment balances the estimated solve cost: the
stage factorization costs about n_s * n_v^2 * (n_v + 8) per step, the step
count grows slowly with the maturity, and a knock-in is two solves (in-out
parity).  Contracts go to ranks longest first, each to the rank with the least
cost so far (longest-processing-time list scheduling), the same rule the
engine uses to order solves over the SMs of one GPU.

The all-gather moves plain tensors (NCCL over NVLink between GPUs, gloo on
CPU); shards are padded to the longest one.  No peer memory is read directly.
"""
from __future__ import annotations

import numpy as np

KNOCK_INS = (0, 1, 4, 5)


def solve_costs(params: np.ndarray, ints: np.ndarray) -> np.ndarray:
    """Estimated relative cost of each contract of a (n, 12) / (n, 3) table."""
    params = np.asarray(params, np.float64)
    ints = np.asarray(ints)
    ns = ints[:, 0].astype(np.float64)
    nv = ints[:, 1].astype(np.float64)
    c = ns * nv * nv * (nv + 8.0) * (1.0 + 0.2 * np.log1p(params[:, 5] / 0.1))
    return c * np.where(np.isin(ints[:, 2], KNOCK_INS), 2.0, 1.0)


def partition(costs: np.ndarray, world: int) -> list[np.ndarray]:
    """Contract indices per rank, ascending within each rank; deterministic,
    so every rank computes the same assignment from the same inputs."""
    costs = np.asarray(costs, np.float64)
    order = np.argsort(-costs, kind="stable")
    load = np.zeros(world)
    owner = np.empty(len(costs), np.int64)
    for j in order:
        r = int(np.argmin(load))  # the first of the least-loaded ranks
        owner[j] = r
        load[r] += costs[j]
    return [np.flatnonzero(owner == r) for r in range(world)]


def gather_prices(local_prices: np.ndarray, local_status: np.ndarray, shards: list[np.ndarray], dist,
                  device) -> tuple[np.ndarray, np.ndarray]:
    """All-gather every rank's (prices, status) of its shard and scatter them
    back into batch order.  Every rank takes this one collective step."""
    import torch

    world = len(shards)
    n = sum(len(s) for s in shards)
    m = max(len(s) for s in shards)
    buf = torch.zeros((2, m), dtype=torch.float64, device=device)
    k = len(local_prices)
    buf[0, :k] = torch.as_tensor(np.asarray(local_prices, np.float64), device=device)
    buf[1, :k] = torch.as_tensor(np.asarray(local_status, np.float64), device=device)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    prices = np.zeros(n)
    status = np.zeros(n, np.int32)
    for r, s in enumerate(shards):
        a = parts[r].cpu().numpy()
        prices[s] = a[0, :len(s)]
        status[s] = a[1, :len(s)].astype(np.int32)
    return prices, status


def price_sharded(params: np.ndarray, ints: np.ndarray, price_fn, dist, device, rank: int,
                  world: int) -> tuple[np.ndarray, np.ndarray]:
    """Price a whole batch across `world` ranks: this rank prices its shard with
    price_fn(params, ints) -> (prices, status), then the gather."""
    shards = partition(solve_costs(params, ints), world)
    mine = shards[rank]
    p, st = price_fn(np.asarray(params)[mine], np.asarray(ints)[mine])
    if world == 1:
        return np.asarray(p, np.float64), np.asarray(st, np.int32)
    return gather_prices(p, st, shards, dist, device)
