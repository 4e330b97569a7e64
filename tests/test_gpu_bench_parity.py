"""Parity on the benchmarked workloads: the CUDA path against the CPU FP64
oracle run now on the same contracts, the same discretization (sinh knots,
span Gauss-Legendre quadrature), the same Radau tolerance and the same
algorithm (direct complex stage solve, exact Radau IIA constants).

- The batched European workload: two contracts of each of the nine grid
  classes (n_s in {32, 48, 64} x n_v in {16, 24, 32}) of the bench's seeded
  256-contract batch.
- The knock-in workload: in-out parity (two solves per price, one on the
  domain truncated at the barrier), eight contracts of the bench's seeded
  barrier batch, grids up to 96 x 48, both solves at 0.01 x rtol.

Relative error = |p - p_oracle| / max(|p_oracle|, 1e-6 S0), the metric's
definition.  Bounds: FP64 factors 1e-6 for Europeans (the same algorithm as
the oracle; their IC projections agree to the ADMM tolerance, and a step
decision that flips on that difference moves a price by a fraction of rtol);
FP32 factors 1e-4 (the metric's gate: the FP32 preconditioner changes the
Newton iterates, so the step sequence and with it the time-discretization
error differ slightly).
"""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

RTOL = 1e-6
FLOOR = 1e-6 * 100.0


def _opts(fpe, precision, **kw):
    return fpe.BatchOptions(disc=1, precision=precision, rtol=RTOL, atol=RTOL * 1e-2, complex_solve=2,
                            radau_constants=2, **kw)


def _oracle(oracle, P, I):
    opt = oracle.options(disc=1, rtol=RTOL, atol=RTOL * 1e-2, complex_direct=1, radau_constants=2)
    return oracle.price_batch(P, I, opt, n_threads=os.cpu_count() or 1)


def _rel(p, ref):
    return np.abs(p - ref) / np.maximum(np.abs(ref), FLOOR)


_BATCH_REF = {}


@pytest.mark.parametrize("block_split", [1, 2])
def test_batched_workload_vs_oracle(engine, oracle, block_split):
    """Both stage-LU block structures (nv x nv blocks, and half-width blocks with
    seven off-diagonal blocks a side) against the same oracle prices."""
    import bench

    fpe = engine
    P, I = bench.make_batch(bench.N_CONTRACTS, 0)
    idx = bench.class_sample(I)
    assert len(idx) == 18
    Ps, Is = P[idx], I[idx]
    if "ref" not in _BATCH_REF:
        _BATCH_REF["ref"] = _oracle(oracle, Ps, Is)
    ref = _BATCH_REF["ref"]
    p64, s64 = fpe.price_batch(Ps, Is, _opts(fpe, 0, block_split=block_split))
    p32, s32 = fpe.price_batch(Ps, Is, _opts(fpe, 1, block_split=block_split))
    assert (s64 == 0).all() and (s32 == 0).all()
    assert _rel(p64, ref).max() < 1e-6, _rel(p64, ref)
    assert _rel(p32, ref).max() < 1e-4, _rel(p32, ref)


def test_knock_in_workload_vs_oracle(engine, oracle):
    """Knock-ins price as vanilla minus knock-out, so the two solves' errors are
    amplified by vanilla / knock-in; on the config discretization both solves
    run at 0.01 x rtol (the default knock_in_tol_scale), and so does the oracle
    here.  The FP64 bound is looser than the Europeans' for the same reason:
    the two implementations make the same discrete decisions (step rejections,
    refactorizations) only up to the IC projection's ADMM tolerance."""
    import bench

    fpe = engine
    P, I = bench.make_barrier_batch(1024, 0)
    big = np.flatnonzero((I[:, 0] == 96) & (I[:, 1] == 48))[:1]
    rest = [j for j in range(0, 1024, 37) if I[j, 0] <= 64 and I[j, 1] <= 32][:7]
    idx = np.concatenate([big, rest]).astype(int)
    assert len(idx) == 8 and set(I[idx, 2]) == {0, 5}
    Ps, Is = P[idx], I[idx]
    opt = oracle.options(disc=1, rtol=RTOL * 0.01, atol=RTOL * 1e-4, complex_direct=1, radau_constants=2)
    ref = oracle.price_batch(Ps, Is, opt, n_threads=os.cpu_count() or 1)
    p64, s64 = fpe.price_batch(Ps, Is, _opts(fpe, 0))
    p32, s32 = fpe.price_batch(Ps, Is, _opts(fpe, 1))
    assert (s64 == 0).all() and (s32 == 0).all()
    assert _rel(p64, ref).max() < 1e-5, _rel(p64, ref)
    assert _rel(p32, ref).max() < 1e-4, _rel(p32, ref)


@pytest.mark.parametrize("block_split", [1, 2])
def test_hard_stage_matrices_vs_oracle(engine, oracle, block_split):
    """The block LU pivots only inside each pivot block (Gauss-Jordan with
    partial pivoting), never across block rows.  The least diagonally dominant
    stage matrices come from low-Feller parameters (2 kappa theta / sigma^2
    well below 1: strong v-diffusion against weak mean reversion), long
    maturities (the largest steps, up to the T/5 cap) and the exact Radau
    constants, factored in FP32.  On such contracts, on the largest config
    grids, the FP32 and FP64 factor paths still match the oracle (which solves
    with pivoted sparse LU) to the workload tolerances."""
    fpe = engine
    rows = []
    for kappa, theta, sigma, rho, T, K in ((0.3, 0.02, 0.9, -0.9, 2.0, 100.0), (0.5, 0.03, 1.0, -0.7, 2.0, 120.0),
                                          (0.2, 0.04, 0.8, 0.0, 1.5, 90.0), (0.4, 0.02, 1.2, -0.5, 2.0, 80.0)):
        assert 2 * kappa * theta / sigma ** 2 < 0.1
        rows.append([kappa, theta, sigma, rho, 0.04, T, 100.0, 0.03, K, 0.0, 0.0, 300.0])
    P = np.array(rows)
    I = np.array([[64, 32, 8], [64, 32, 9], [48, 24, 8], [64, 24, 9]], np.int32)
    ref = _oracle(oracle, P, I)
    p64, s64 = fpe.price_batch(P, I, _opts(fpe, 0, block_split=block_split))
    p32, s32 = fpe.price_batch(P, I, _opts(fpe, 1, block_split=block_split))
    assert (s64 == 0).all() and (s32 == 0).all(), (s64, s32)
    assert _rel(p64, ref).max() < 1e-6, _rel(p64, ref)
    assert _rel(p32, ref).max() < 1e-4, _rel(p32, ref)
