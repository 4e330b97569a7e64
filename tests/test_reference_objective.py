"""The reference calibrator's objective (src/engines/calibrator/objective.mojo:
26-104): per quote an FPE solve on the reference discretization with 8 x 8
knots, 251 grid inserts, FPESolver(rtol 1e-5, atol 1e-7, max_step 0.02,
first_step 0 = the Radau solver's own first step, radau.mojo:168-184), and
the objective's own density integration: payoff x pdf x half the neighbour
spacing in s and v (1 at both ends), undiscounted (:26-50).

CPU: the oracle's integration rule against a numpy restatement of :26-50 on
the oracle's own pdf and quadrature points.  GPU: the device solve with the
same options against the oracle (FP64, GMRES(10), the reference's Radau
constants, so the two follow the same step sequence), and the LM calibrator
on quotes made by the same objective.
"""
import numpy as np
import pytest

H = dict(kappa=1.2, theta=0.05, sigma=0.35, rho=-0.4, r=0.1, T=0.6, S0=60.0, V0=0.1)
KS = [55.0, 60.0, 70.0]


def _oracle_opts(oracle, first_step=-1.0, price_rule=1):
    return oracle.options(disc=0, num_insert=251, rtol=1e-5, atol=1e-7, max_step=0.02,
                          first_step=first_step, price_rule=price_rule)


def test_oracle_objective_integration_matches_its_formula(oracle):
    pl = oracle.Pipeline(**H, n_s=8, n_v=8, option_type=8, s_max=180.0, opt=_oracle_opts(oracle))
    got = pl.price_at(KS)
    s, v = pl.array("s"), pl.array("v")
    pdf = pl.array("pdf").reshape(len(s), len(v))
    ds = np.ones(len(s))
    ds[1:-1] = 0.5 * (s[2:] - s[:-2])
    dv = np.ones(len(v))
    dv[1:-1] = 0.5 * (v[2:] - v[:-2])
    ref = [float(np.sum(np.maximum(s - K, 0.0)[:, None] * pdf * ds[:, None] * dv[None, :])) for K in KS]
    np.testing.assert_allclose(got, ref, rtol=1e-12)
    # the solver's own first step changes the step sequence, not the solution
    alt = oracle.Pipeline(**H, n_s=8, n_v=8, option_type=8, s_max=180.0,
                          opt=_oracle_opts(oracle, first_step=0.0)).price_at(KS)
    np.testing.assert_allclose(got, alt, rtol=1e-4)


def _tables(rows):
    P = np.array([[*h, k, 0.0, 0.0, 3.0 * h[6]] for h, k in rows])
    I = np.array([[8, 8, 8]] * len(rows), np.int32)
    return P, I


@pytest.mark.gpu
def test_device_objective_prices_match_oracle(engine, oracle):
    fpe = engine
    h2 = (1.8, 0.07, 0.5, -0.6, 0.03, 1.2, 100.0, 0.06)
    rows = [(tuple(H.values()), k) for k in KS] + [(h2, k) for k in (90.0, 100.0, 115.0)]
    P, I = _tables(rows)
    opts = fpe.BatchOptions(disc=0, precision=0, num_insert=251, rtol=1e-5, atol=1e-7, complex_solve=1,
                            radau_constants=1, max_step=0.02, first_step=-1.0, price_rule=1)
    got, st = fpe.price_batch(P, I, opts)
    assert (st == 0).all()
    ref = oracle.price_batch(P, I, _oracle_opts(oracle), n_threads=6)
    print("objective prices", got, "oracle", ref)
    np.testing.assert_allclose(got, ref, rtol=1e-8, atol=1e-10)
    # the rule differs from the Pricer's (discounted quadrature) on the same solve
    pr, _ = fpe.price_batch(P, I, fpe.BatchOptions(disc=0, precision=0, num_insert=251, rtol=1e-5,
                                                   atol=1e-7, complex_solve=1, radau_constants=1,
                                                   max_step=0.02, first_step=-1.0))
    ref0 = oracle.price_batch(P, I, _oracle_opts(oracle, price_rule=0), n_threads=6)
    np.testing.assert_allclose(pr, ref0, rtol=1e-8, atol=1e-10)
    assert np.all(np.abs(pr - got) > 1e-3)


@pytest.mark.gpu
def test_reference_calibrator_on_its_own_objective(engine):
    from fpe_option_b200.calibration import ReferenceObjectiveSurface, Surface, calibrate_reference_objective

    truth = np.array([1.5, 0.06, 0.4, -0.5, 0.05])
    surf = Surface.grid(100.0, 0.02, [0.9, 1.0, 1.1], [0.5, 1.0])
    surf.prices = ReferenceObjectiveSurface(surf).price_sets(np.atleast_2d(truth))[0]
    x0 = truth * np.array([1.1, 0.9, 1.1, 0.9, 1.1])
    be = ReferenceObjectiveSurface(surf)
    r0 = be.residual(x0)
    x, info = calibrate_reference_objective(surf, x0, max_iter=25)
    r1 = ReferenceObjectiveSurface(surf).residual(x)
    print("reference calibrator:", info, "x", x, "truth", truth,
          "cost %.3e -> %.3e" % (float(r0 @ r0), float(r1 @ r1)))
    assert float(r1 @ r1) < 1e-2 * float(r0 @ r0)
