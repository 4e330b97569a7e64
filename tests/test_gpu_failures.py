"""Failure handling of the batched solve on the GPU: every status word the
kernels can write is provoked on the host side (options and inputs), never by
a fault.  The reference ends a Radau solve with "max steps exceeded" and
"step size underflow" (src/numerics/ode/radau.mojo:257-263, :274-281,
:458-464); the batch reports them per solve as status codes.

- FPE_STATUS_MAX_STEPS: max_steps=3 caps the accepted steps.
- FPE_STATUS_STEP_UNDERFLOW: a maturity of 1e-15 years asks for a first step
  below the 1e-14 floor.
- FPE_STATUS_SINGULAR: sigma = 1e200 overflows the stiffness factors to Inf,
  so the first stage factorization meets a non-finite pivot and the solve
  stops there.
- FPE_STATUS_TIMEOUT: stage_wait_cycles=1 makes the staged sweep's bounded
  wait on its bulk copies give up at once; the copies still in flight are
  waited out with the full limit before the solve ends.
- FPE_STATUS_INVALID: NaN / Inf parameters are rejected on the host.
- The FP64 retry: a mixed-precision solve that fails is solved again with FP64
  factors, and its price then equals the FP64 plan's.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROW = [1.2, 0.05, 0.35, -0.4, 0.03, 0.6, 100.0, 0.1, 100.0, 0.0, 0.0, 300.0]
MAX_STEPS, STEP_UNDERFLOW, SINGULAR, TIMEOUT, INVALID = 4, 5, 3, 7, 16


def _batch(rows, grid=(24, 16), otype=8):
    P = np.array(rows, dtype=np.float64)
    I = np.tile(np.array([[grid[0], grid[1], otype]], np.int32), (len(P), 1))
    return P, I


def _opts(fpe, precision=1, **kw):
    base = dict(disc=1, precision=precision, rtol=1e-6, atol=1e-8, complex_solve=2, radau_constants=2)
    base.update(kw)
    return fpe.BatchOptions(**base)


def _plan(fpe, P, I, opts):
    arr, keep = fpe.contracts_from_arrays(P, I)
    plan = fpe.Plan(arr, opts, _keep=keep)
    plan.run()
    p, _, _, _, st = plan.results()
    n = plan.retried()
    plan.close()
    return p, st, n


@pytest.mark.parametrize("precision", [0, 1])
def test_max_steps(engine, precision):
    fpe = engine
    P, I = _batch([ROW, ROW])
    p, st, _ = _plan(fpe, P, I, _opts(fpe, precision, max_steps=3))
    assert (st == MAX_STEPS).all(), st
    # the cap does not touch a solve that needs fewer steps
    p2, st2, _ = _plan(fpe, P, I, _opts(fpe, precision, max_steps=100000))
    p3, st3, _ = _plan(fpe, P, I, _opts(fpe, precision))
    assert (st2 == 0).all() and (st3 == 0).all()
    assert np.array_equal(p2, p3)


def test_step_underflow(engine):
    fpe = engine
    row = list(ROW)
    row[5] = 1e-15
    P, I = _batch([row])
    for precision in (0, 1):
        _, st, _ = _plan(fpe, P, I, _opts(fpe, precision))
        assert st[0] == STEP_UNDERFLOW, st


def test_singular_factor_ends_the_solve(engine):
    fpe = engine
    row = list(ROW)
    row[2] = 1e200  # sigma: the stiffness factors overflow to Inf
    P, I = _batch([row, ROW])
    for precision in (0, 1):
        p, st, _ = _plan(fpe, P, I, _opts(fpe, precision))
        assert st[0] == SINGULAR, st
        assert st[1] == 0 and np.isfinite(p[1])  # the other solve of the batch is unaffected


def test_invalid_nonfinite_parameters(engine):
    fpe = engine
    rows = []
    for k in (0, 1, 2, 3, 4, 5, 6, 7, 8, 11):
        for bad in ((np.inf,) if k == 11 else (np.nan, np.inf)):  # s_max NaN means "3 S0"
            r = list(ROW)
            r[k] = bad
            rows.append(r)
    rows.append(ROW)
    P, I = _batch(rows)
    p, st, _ = _plan(fpe, P, I, _opts(fpe, 1))
    assert (st[:-1] == INVALID).all(), st
    assert st[-1] == 0 and np.isfinite(p[-1])


def test_stage_wait_timeout_and_fp64_retry(engine):
    fpe = engine
    P, I = _batch([ROW, [2.0, 0.08, 0.5, -0.6, 0.01, 1.2, 100.0, 0.05, 95.0, 0.0, 0.0, 300.0]])
    # a one-cycle wait gives up on the first stage whose copies have not landed
    _, st, n = _plan(fpe, P, I, _opts(fpe, 1, stage_wait_cycles=1, fp64_retry=-1))
    assert (st == TIMEOUT).all(), st
    assert n == 0
    # the same failure, re-solved with FP64 factors (default wait) by the retry
    p, st, n = _plan(fpe, P, I, _opts(fpe, 1, stage_wait_cycles=1))
    assert (st == 0).all(), st
    assert n == 2
    p64, st64, _ = _plan(fpe, P, I, _opts(fpe, 0))
    assert (st64 == 0).all()
    assert np.allclose(p, p64, rtol=1e-12, atol=0.0), (p, p64)
    # the library keeps working after the timeouts
    p1, st1, n1 = _plan(fpe, P, I, _opts(fpe, 1))
    assert (st1 == 0).all() and n1 == 0
    assert np.allclose(p1, p64, rtol=1e-5)


def test_retry_keeps_a_failure_the_fp64_solve_shares(engine):
    """max_steps applies to the FP64 attempt too: the retry runs, and the
    status of its attempt is reported."""
    fpe = engine
    P, I = _batch([ROW])
    _, st, n = _plan(fpe, P, I, _opts(fpe, 1, max_steps=3))
    assert st[0] == MAX_STEPS and n == 1
