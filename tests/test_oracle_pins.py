"""The CPU oracle against every published number and component test of the
reference (elevenwang-creator/FPE_option), and against the committed golden
fixtures.  CPU only."""
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "oracle_golden.json")
H = dict(kappa=1.2, theta=0.05, sigma=0.35, rho=-0.4, r=0.1, T=0.6, S0=60.0, V0=0.1)


def test_readme_european_prices_and_greeks(oracle):
    # README.md:380-392: price(n_s=n_v=38, K=[80,90,100], s_max=150, european_call)
    p, d, g, v, rc = oracle.engine_price(*H.values(), K=[80, 90, 100], option_type=8, n_s=38,
                                         n_v=38, s_max=150.0)
    assert rc == 0
    np.testing.assert_allclose(p, [0.966276, 0.280919, 0.078883], atol=6e-7)
    np.testing.assert_allclose(d, [0.175855, 0.060298, 0.018875], atol=6e-7)
    np.testing.assert_allclose(g, [0.017766, 0.009270, 0.002742], atol=6e-7)
    np.testing.assert_allclose(v, [14.057144, 6.197252, 2.283113], atol=6e-6)


def test_readme_down_and_out_prices(oracle):
    # README.md:397-404
    p = oracle.pricer_price(*H.values(), K=[80, 90, 100], barrier=50.0, option_type=2, n_s=38,
                            n_v=38, s_max=150.0)
    np.testing.assert_allclose(p, [0.905038, 0.263874, 0.074223], atol=6e-7)


@pytest.mark.parametrize("ot,expected", [
    (2, [4.4383, 2.7694, 1.6319, 0.9195, 0.5023, 0.2692, 0.1430, 0.0758]),  # README.md:657-668 DOC
    (8, [4.6762, 2.8855, 1.6881, 0.9468, 0.5155, 0.2758, 0.1463, 0.0774]),  # README.md:672-683 vanilla
    (0, [0.2379, 0.1161, 0.0562, 0.0272, 0.0133, 0.0065, 0.0033, 0.0017]),  # README.md:672-683 DIC
])
def test_readme_num_insert_251_tables(oracle, ot, expected):
    K = [65, 70, 75, 80, 85, 90, 95, 100]
    p = oracle.pricer_price(*H.values(), K=K, barrier=0.0 if ot == 8 else 50.0, option_type=ot,
                            n_s=38, n_v=38, s_max=150.0, opt=oracle.options(num_insert=251))
    np.testing.assert_allclose(p, expected, atol=5.1e-5)


def test_bspline_values_and_partition_of_unity(oracle):
    # tests/test_bspline.mojo:16-40
    knots = [0.0, 0.0, 0.5, 1.0, 1.0]
    assert abs(oracle.bspline_value(knots, 1, 0.25, 0) - 0.5) < 1e-10
    assert abs(oracle.bspline_value(knots, 1, 0.25, 1) - 0.5) < 1e-10
    assert abs(oracle.bspline_value(knots, 1, 0.25, 2) - 0.0) < 1e-10
    assert abs(oracle.bspline_value(knots, 1, 0.75, 1) - 0.5) < 1e-10
    assert abs(oracle.bspline_value(knots, 1, 0.75, 2) - 0.5) < 1e-10
    for x in [0.1, 0.25, 0.5, 0.75, 0.9]:
        assert abs(sum(oracle.bspline_value(knots, 1, x, i) for i in range(3)) - 1.0) < 1e-10
    cub = [0, 0, 0, 0, 0.2, 0.5, 0.7, 1, 1, 1, 1]
    for x in np.linspace(0.0, 0.999, 37):
        assert abs(sum(oracle.bspline_value(cub, 3, x, i) for i in range(7)) - 1.0) < 1e-12


def test_uniform_knots_repeat_boundaries(oracle):
    # tests/test_bspline.mojo:43-59
    k = oracle.generate_knots(8, 2, False, 0.2, 0.0, 1.0, 50.0, 0.1)
    assert len(k) == 8
    assert abs(k[0]) < 1e-10 and abs(k[1]) < 1e-10
    assert abs(k[6] - 1) < 1e-10 and abs(k[7] - 1) < 1e-10


@pytest.mark.parametrize("ot,K,B,S,exp", [  # tests/test_barrier_payoff.mojo:18-120
    (0, 100.0, 80.0, 70.0, 0.0), (0, 100.0, 80.0, 90.0, 0.0), (0, 100.0, 80.0, 60.0, 0.0),
    (2, 100.0, 80.0, 120.0, 20.0), (2, 100.0, 80.0, 70.0, 0.0), (6, 100.0, 120.0, 110.0, 10.0),
    (6, 100.0, 120.0, 130.0, 0.0), (5, 100.0, 120.0, 130.0, 0.0), (5, 100.0, 120.0, 90.0, 0.0),
    (8, 100.0, 0.0, 120.0, 20.0), (8, 100.0, 0.0, 80.0, 0.0), (9, 100.0, 0.0, 80.0, 20.0),
    (9, 100.0, 0.0, 120.0, 0.0), (1, 100.0, 80.0, 70.0, 30.0), (3, 100.0, 80.0, 90.0, 10.0),
    (4, 100.0, 120.0, 125.0, 25.0), (7, 100.0, 120.0, 90.0, 10.0),
])
def test_barrier_payoff_values(oracle, ot, K, B, S, exp):
    assert abs(oracle.payoff(ot, [K], B, S)[0] - exp) < 1e-12


@pytest.mark.parametrize("M,Kd,y0", [  # tests/test_radau.mojo:72-160
    (np.eye(3), np.diag([1.0, 2.0, 3.0]), np.ones(3)),
    (np.diag([2.0, 3.0, 4.0]), np.diag([1.0, 2.0, 3.0]), np.ones(3)),
])
def test_radau_exponential_decay(oracle, M, Kd, y0):
    y, n = oracle.radau_dense(M, Kd, y0, 1.0, 1e-3, 1e-6, 0.0, 0.1)
    exact = y0 * np.exp(-np.diag(Kd) / np.diag(M))
    assert n > 0
    assert np.max(np.abs(y - exact)) < 1e-3


def _dense_problem():
    from scipy.linalg import expm, solve

    rng = np.random.default_rng(3)
    A = rng.standard_normal((6, 6))
    Kd = A @ A.T + 6 * np.eye(6)
    M = np.eye(6) + 0.1 * np.diag(rng.random(6))
    y0 = rng.standard_normal(6)
    return M, Kd, y0, expm(-0.7 * solve(M, Kd)) @ y0


def test_radau_exact_constants_converge_at_order_five(oracle):
    """With the true Radau IIA eigenvalues (and TI13 = inv(T)[0][2]) the error
    falls with the tolerance and the step count grows slowly."""
    M, Kd, y0, exact = _dense_problem()
    errs, steps = [], []
    for rt in (1e-4, 1e-6, 1e-8, 1e-10):
        y, n = oracle.radau_dense(M, Kd, y0, 0.7, rt, rt * 1e-2, 0.0, 1e-6, exact=True)
        errs.append(np.max(np.abs(y - exact)))
        steps.append(n)
    assert errs[-1] < 1e-9 and errs[0] > errs[-1] * 100
    assert all(0 < s < 400 for s in steps)


def test_radau_reference_constants_error_floor(oracle):
    """The reference's hard-coded U1/ALPH/BETA/TI13 (radau.mojo:64-75) are not the
    Radau IIA values; its error stalls near 1e-5 however tight the tolerance,
    while the step count explodes.  The oracle reproduces that behaviour."""
    M, Kd, y0, exact = _dense_problem()
    y4, n4 = oracle.radau_dense(M, Kd, y0, 0.7, 1e-4, 1e-6, 0.0, 1e-6)
    y8, n8 = oracle.radau_dense(M, Kd, y0, 0.7, 1e-8, 1e-10, 0.0, 1e-6)
    e4, e8 = np.max(np.abs(y4 - exact)), np.max(np.abs(y8 - exact))
    assert 1e-6 < e8 < 1e-4 and 1e-6 < e4 < 1e-4
    assert n8 > 50 * n4


def test_heston_cf_put_call_parity_and_fpe(oracle):
    c = oracle.heston_cf(*H.values(), K=80.0, is_call=True)
    p = oracle.heston_cf(*H.values(), K=80.0, is_call=False)
    assert abs((c - p) - (60.0 - 80.0 * np.exp(-0.1 * 0.6))) < 1e-10
    assert 0.0 < c < 60.0
    # the FPE price on the reference discretization agrees to its discretization error
    fpe = oracle.pricer_price(*H.values(), K=[80.0], option_type=8, n_s=38, n_v=38,
                              s_max=150.0)[0]
    assert abs(fpe - c) / c < 0.05


def test_golden_fixtures(oracle):
    """The oracle reproduces the committed fixtures (made by tests/golden/make_golden.py)."""
    with open(GOLDEN) as f:
        gold = json.load(f)
    for case in gold["small_cases"]:
        args = case["args"]
        opt = oracle.options(**case.get("options", {}))
        p = oracle.pricer_price(**args, opt=opt)
        np.testing.assert_allclose(p, case["prices"], rtol=1e-11, atol=1e-14)


@pytest.mark.parametrize("ns,nv,T,V0", [(24, 16, 0.6, 0.1), (32, 24, 1.2, 0.05), (40, 24, 0.3, 0.02)])
def test_config_ic_admm_reaches_the_exact_projection(oracle, ns, nv, T, V0):
    """The config discretization's IC ADMM (residual-balanced rho, over-
    relaxation 1.6) converges to the nonnegative least-squares projection that
    the exact active-set solver finds, to the ADMM's 1e-8 residual scale."""
    h = dict(H, T=T, V0=V0)
    kw = dict(n_s=ns, n_v=nv, option_type=8, s_max=180.0)
    pa = oracle.Pipeline(**h, **kw, opt=oracle.options(disc=1))
    qa = pa.array("q0")
    qe = oracle.Pipeline(**h, **kw, opt=oracle.options(disc=1, nnls_exact=1)).array("q0")
    assert np.linalg.norm(qa - qe) <= 1e-6 * np.linalg.norm(qe)
    assert pa.dims()["admm"] < 500
