"""Heston characteristic-function prices of Europeans.

CPU: the oracle's price (Heston 1993 probabilities P1, P2 in the Albrecher et
al. 2007 form, composite Gauss-Legendre) against an independent formulation,
Lewis's (2001) single integral of the characteristic function of ln(S_T/F)
along Im u = -1/2, integrated by adaptive quadrature (scipy); that integrator
is itself checked on the Black-Scholes characteristic function against the
closed form.  The reference engine has no closed-form price to pin against.

GPU: the device kernel (fpe_heston_cf_batch / fpe_heston_cf_price) against
the oracle on the same inputs.  Both run the same quadrature in FP64; they
differ in the order of the 16-node panel sums and in the last bits of the
device's transcendental functions, so prices agree to 1e-11 relative plus
1e-12 S0 absolute (the call is S0 P1 - K e^{-rT} P2, a difference of two
numbers of order S0).
"""
import ctypes as C

import numpy as np
import pytest

H = dict(kappa=1.2, theta=0.05, sigma=0.35, rho=-0.4, r=0.1, T=0.6, S0=60.0, V0=0.1)


def _lewis_call(phi, S0, K, r, T):
    from scipy.integrate import quad

    k = np.log(S0 / K) + r * T
    f = lambda u: (np.exp(1j * u * k) * phi(u - 0.5j)).real / (u * u + 0.25)
    val, _ = quad(f, 0.0, np.inf, limit=2000, epsabs=1e-13, epsrel=1e-12)
    return S0 - np.sqrt(S0 * K) * np.exp(-0.5 * r * T) / np.pi * val


def _heston_phi(kappa, theta, sigma, rho, T, V0):
    """Characteristic function of ln(S_T / F_T) under Heston (Gatheral's form)."""

    def phi(u):
        b = kappa - rho * sigma * 1j * u
        d = np.sqrt(b * b + sigma ** 2 * (u * u + 1j * u))
        g = (b - d) / (b + d)
        e = np.exp(-d * T)
        A = kappa * theta / sigma ** 2 * ((b - d) * T - 2.0 * np.log((1.0 - g * e) / (1.0 - g)))
        B = (b - d) / sigma ** 2 * (1.0 - e) / (1.0 - g * e)
        return np.exp(A + B * V0)

    return phi


def _draw(n, seed, S0=100.0):
    """Random parameter rows (kappa theta sigma rho r T S0 V0), strikes, put flags."""
    rng = np.random.default_rng(seed)
    P = np.column_stack([rng.uniform(0.5, 3.0, n), rng.uniform(0.02, 0.12, n),
                         rng.uniform(0.1, 0.8, n), rng.uniform(-0.9, 0.3, n),
                         rng.uniform(0.0, 0.1, n), rng.uniform(0.1, 2.0, n), np.full(n, S0),
                         rng.uniform(0.01, 0.15, n)])
    K = S0 * rng.uniform(0.7, 1.4, n)
    put = (rng.uniform(size=n) < 0.5).astype(np.int32)
    return P, K, put


def test_lewis_integrator_reproduces_black_scholes():
    from scipy.stats import norm

    S0, r, T, vol = 60.0, 0.1, 0.6, 0.3
    for K in (40.0, 60.0, 90.0):
        d1 = (np.log(S0 / K) + (r + 0.5 * vol * vol) * T) / (vol * np.sqrt(T))
        bs = S0 * norm.cdf(d1) - K * np.exp(-r * T) * norm.cdf(d1 - vol * np.sqrt(T))
        got = _lewis_call(lambda u: np.exp(-0.5 * vol * vol * T * (u * u + 1j * u)), S0, K, r, T)
        assert abs(got - bs) < 1e-11


def test_oracle_cf_matches_lewis_formulation(oracle):
    P, K, _ = _draw(12, seed=0)
    for p, k in zip(P, K):
        a = oracle.heston_cf(*p, k, True)
        b = _lewis_call(_heston_phi(p[0], p[1], p[2], p[3], p[5], p[7]), p[6], k, p[4], p[5])
        assert abs(a - b) < 1e-10 * p[6], (p, k, a, b)
    # the README parameter set, strikes either side of the money
    for k in (50.0, 60.0, 80.0):
        a = oracle.heston_cf(*H.values(), k, True)
        b = _lewis_call(_heston_phi(1.2, 0.05, 0.35, -0.4, 0.6, 0.1), 60.0, k, 0.1, 0.6)
        assert abs(a - b) < 1e-10 * 60.0


def _oracle_prices(oracle, P, K, put):
    return np.array([oracle.heston_cf(*p, k, not q) for p, k, q in zip(P, K, put)])


@pytest.mark.gpu
def test_device_cf_matches_oracle(engine, oracle):
    import torch

    from fpe_option_b200 import _lib

    L = _lib.load()
    P, K, put = _draw(256, seed=3)
    # slowly decaying integrands: short maturities, low variance (many panels)
    Q, KQ, putQ = _draw(32, seed=4)
    Q[:, 5] = np.linspace(0.02, 0.1, 32)
    Q[:, 7] = np.linspace(0.002, 0.02, 32)
    Q[:, 2] = np.linspace(0.05, 1.5, 32)
    P, K, put = np.vstack([P, Q]), np.concatenate([K, KQ]), np.concatenate([put, putQ])
    ref = _oracle_prices(oracle, P, K, put)
    tP = torch.tensor(P, device="cuda")
    tK = torch.tensor(K, device="cuda")
    tput = torch.tensor(put, device="cuda")
    out = torch.full((len(K),), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream or 1
    rc = L.fpe_heston_cf_batch(tP.data_ptr(), tK.data_ptr(), tput.data_ptr(), len(K),
                               out.data_ptr(), stream)
    assert rc == 0
    got = out.cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-12 * 100.0)
    # NULL put flags: all calls
    rc = L.fpe_heston_cf_batch(tP.data_ptr(), tK.data_ptr(), None, len(K), out.data_ptr(), stream)
    assert rc == 0
    calls = out.cpu().numpy()
    ref_c = _oracle_prices(oracle, P, K, np.zeros_like(put))
    np.testing.assert_allclose(calls, ref_c, rtol=1e-11, atol=1e-12 * 100.0)
    # put-call parity on the device values
    disc = K * np.exp(-P[:, 4] * P[:, 5])
    m = put == 1
    np.testing.assert_allclose(calls[m] - got[m], P[m, 6] - disc[m], rtol=0, atol=1e-11 * 100.0)


@pytest.mark.gpu
def test_device_cf_argument_and_domain_errors(engine):
    import torch

    from fpe_option_b200 import _lib

    L = _lib.load()
    P = torch.tensor([[1.2, 0.05, 0.35, -0.4, 0.1, 0.6, 60.0, 0.1],
                      [1.2, 0.05, -0.35, -0.4, 0.1, 0.6, 60.0, 0.1],  # sigma < 0
                      [1.2, 0.05, 0.35, -1.4, 0.1, 0.6, 60.0, 0.1],   # |rho| > 1
                      [1.2, 0.05, 0.35, -0.4, 0.1, 0.6, 60.0, float("nan")]], dtype=torch.float64,
                     device="cuda")
    K = torch.tensor([60.0, 60.0, 60.0, 60.0], dtype=torch.float64, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    assert L.fpe_heston_cf_batch(P.data_ptr(), K.data_ptr(), None, 4, out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    assert np.isfinite(o[0]) and np.isnan(o[1:]).all()
    assert L.fpe_heston_cf_batch(P.data_ptr(), K.data_ptr(), None, 0, out.data_ptr(), None) == 0
    assert L.fpe_heston_cf_batch(P.data_ptr(), K.data_ptr(), None, -1, out.data_ptr(), None) < 0
    assert L.fpe_heston_cf_batch(None, K.data_ptr(), None, 4, out.data_ptr(), None) < 0


@pytest.mark.gpu
def test_host_entry_point_statuses_and_fpe_discretization_error(engine, oracle):
    fpe = engine
    S0 = 60.0
    K = [48.0, 54.0, 60.0, 66.0, 75.0]
    rows = []
    for ot in (8, 9):
        for k in K:
            rows.append([1.2, 0.05, 0.35, -0.4, 0.1, 0.6, S0, 0.1, k, 0.0, 0.0, 180.0])
    P = np.array(rows)
    I = np.array([[40, 24, 8]] * 5 + [[40, 24, 9]] * 5, np.int32)
    cf, st = fpe.heston_cf_price(P, I)
    assert (st == 0).all()
    ref = np.array([oracle.heston_cf(*p[:8], p[8], i[2] == 8) for p, i in zip(P, I)])
    np.testing.assert_allclose(cf, ref, rtol=1e-11, atol=1e-12 * S0)
    # the FPE prices of the same contracts (config discretization, 40 x 24) sit
    # within their discretization error of the closed-form value
    got, st2 = fpe.price_batch(P, I, fpe.BatchOptions(disc=1, precision=0, rtol=1e-8, atol=1e-10,
                                                     complex_solve=2, radau_constants=2))
    assert (st2 == 0).all()
    err = np.abs(got - cf) / (cf + 1e-2 * S0)
    print("FPE vs CF relative deviation:", np.array2string(err, precision=2))
    assert err.max() < 2e-2
    # barrier types are not priced; invalid strikes are flagged
    B = P[:2].copy()
    B[0, 9] = 50.0
    B[1, 8] = -1.0
    p2, st3 = fpe.heston_cf_price(B, np.array([[40, 24, 2], [40, 24, 8]], np.int32))
    assert st3[0] == 2 and st3[1] == 16 and np.isnan(p2).all()
