"""The learned part end to end, on a reduced scale that runs in seconds:
FPE prices train the tensor-core ensemble, held-out quotes are judged by the
FPE solver, untrusted queries fall back to it, the network answers held-out
queries at a stated error thousands of times faster than the solver (the gain
it brings), and a calibration with the surrogate in the loop followed by an
FPE polish reaches the FPE-only fit.  (Whether surrogate-in-loop calibration
also saves FPE solves depends on the surrogate's accuracy, which needs the
full-size training set; bench.py --workload calibration measures it.)"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRID = (32, 16)


@pytest.fixture(scope="module")
def trained(engine):
    from fpe_option_b200 import BatchOptions
    from fpe_option_b200.surrogate import SurrogateConfig, SurrogatePricer, draw_contracts

    opts = BatchOptions(disc=1, precision=1, rtol=1e-6, atol=1e-8, complex_solve=2, radau_constants=2)
    # a small training set: members agree to a few percent, so the trust
    # tolerance is 5e-2 here (the full-size surrogate uses 1e-3)
    pr = SurrogatePricer(SurrogateConfig(members=3, batch=1024, epochs=120, seed=1, disagreement_tol=5e-2),
                         fpe_options=opts)
    P, I = draw_contracts(16384, seed=10, kind="european", grid=GRID)
    y = pr.fpe_prices(P, I)
    losses = pr.fit(P, I, y)
    yield pr, losses
    pr.close()


def test_held_out_quotes_judged_by_fpe(trained):
    from fpe_option_b200.surrogate import draw_contracts, encode

    pr, losses = trained
    P, I = draw_contracts(512, seed=99, kind="european", grid=GRID)
    ref = pr.fpe_prices(P, I)
    import torch

    x, _ = encode(P, I)
    mean, spread = pr.predict_features(torch.as_tensor(x, device="cuda"))
    got = pr.to_price(mean.cpu().numpy(), P, I)
    rel = np.abs(got - ref) / (np.abs(ref) + 0.2)  # 0.2 = 2e-3 S0 price floor
    print("held-out rel err: median %.2e p90 %.2e max %.2e; losses %s"
          % (np.median(rel), np.quantile(rel, 0.9), rel.max(), losses))
    assert np.median(rel) < 3e-2
    assert np.quantile(rel, 0.9) < 1e-1


def test_untrusted_queries_fall_back_to_fpe(trained):
    from fpe_option_b200.surrogate import draw_contracts

    pr, _ = trained
    P, I = draw_contracts(8, seed=5, kind="european", grid=GRID)
    P[:4, 0] = 5.0  # kappa outside the training box
    I[6, 2] = 3     # down-and-out put: an option type the surrogate does not cover
    P[6, 9] = 80.0
    prices, fb = pr.price(P, I)
    assert fb[:4].all() and fb[6]
    ref = pr.fpe_prices(P[fb], I[fb])
    assert np.array_equal(prices[fb], ref)  # answered by the solver itself


def test_surrogate_throughput_gain_at_stated_error(trained):
    import time

    import torch

    from fpe_option_b200.surrogate import draw_contracts, encode

    pr, _ = trained
    P, I = draw_contracts(256, seed=123, kind="european", grid=GRID)
    t0 = time.perf_counter()
    ref = pr.fpe_prices(P, I)
    fpe_rate = len(P) / (time.perf_counter() - t0)
    Q, J = draw_contracts(65536, seed=124, kind="european", grid=GRID)
    x = torch.as_tensor(encode(Q, J)[0], device="cuda")
    pr.predict_features(x)  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pr.predict_features(x)
    torch.cuda.synchronize()
    sur_rate = len(Q) / (time.perf_counter() - t0)
    xs = torch.as_tensor(encode(P, I)[0], device="cuda")
    got = pr.to_price(pr.predict_features(xs)[0].cpu().numpy(), P, I)
    rel = np.abs(got - ref) / (np.abs(ref) + 0.2)
    print("FPE %.0f prices/s, surrogate (3 members) %.3e prices/s, ratio %.0f, median rel err %.2e"
          % (fpe_rate, sur_rate, sur_rate / fpe_rate, np.median(rel)))
    assert sur_rate > 300.0 * fpe_rate
    assert np.median(rel) < 3e-2


def test_surrogate_then_fpe_polish_reaches_the_fpe_fit(trained):
    from fpe_option_b200 import BatchOptions, price_batch
    from fpe_option_b200.calibration import Surface, calibrate_fpe, calibrate_with_surrogate, contract_tables

    pr, _ = trained
    truth = np.array([1.6, 0.07, 0.45, -0.55, 0.08])
    surf = Surface.grid(100.0, 0.02, [0.85, 0.95, 1.0, 1.05, 1.15], [0.4, 0.9, 1.5])
    P, I = contract_tables(surf, truth, GRID)
    p, st = price_batch(P, I, BatchOptions(disc=1, precision=0, rtol=1e-9, atol=1e-11,
                                           complex_solve=2, radau_constants=2))
    assert (st == 0).all()
    surf.prices = p
    x0 = np.array([1.0, 0.05, 0.3, -0.3, 0.05])
    kw = {"grid": GRID}
    x_f, info_f = calibrate_fpe(surf, x0, **kw)
    x_s, info_s = calibrate_with_surrogate(surf, pr, x0, max_iter=30, polish_iter=30, fpe_kw=kw)
    x_p, info_p = calibrate_with_surrogate(surf, pr, x0, max_iter=30, polish="fpe", polish_iter=30, fpe_kw=kw)
    assert np.abs(x_p - truth).max() / 1.0 < 1e-3
    err_f = np.abs(x_f - truth) / np.abs(truth)
    err_s = np.abs(x_s - truth) / np.abs(truth)
    print("fpe-only", info_f, err_f, "\nsurrogate+hybrid polish", info_s, err_s, "\n+fpe polish", info_p)
    assert err_f.max() < 1e-4
    # the hybrid polish (FPE residuals, surrogate Jacobians) lowers the FPE residual
    from fpe_option_b200.calibration import FpeSurface

    fb = FpeSurface(surf, grid=GRID)
    r_fit = fb.residual(np.array(info_s["x_surrogate_fit"]))
    r_pol = fb.residual(x_s)
    assert float(r_pol @ r_pol) < float(r_fit @ r_fit)
