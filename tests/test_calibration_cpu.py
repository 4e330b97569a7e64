"""CPU checks of the Levenberg-Marquardt restatement (reference
src/numerics/optim/lm.mojo:29-121) and the calibrator clamps
(src/engines/calibrator/calibrator.mojo:15-29)."""
import numpy as np
import pytest

from fpe_option_b200.calibration import Surface, clamp, contract_tables, levenberg_marquardt


def test_lm_solves_a_curve_fit():
    t = np.linspace(0, 1, 30)
    a_true = np.array([2.0, -1.3, 0.4])
    y = a_true[0] * np.exp(a_true[1] * t) + a_true[2]

    def res(a):
        return a[0] * np.exp(a[1] * t) + a[2] - y

    def jac(a):
        e = np.exp(a[1] * t)
        return res(a), np.stack([e, a[0] * t * e, np.ones_like(t)], axis=1)

    out = levenberg_marquardt(res, jac, np.array([1.0, 0.0, 0.0]), max_iter=100, tol=1e-12)
    assert np.allclose(out.x, a_true, atol=1e-8)


def test_lm_damping_rises_on_rejected_steps():
    # a step that increases the cost is rejected and lambda grows tenfold
    def res(x):
        return np.array([x[0] ** 2 - 1e-3])

    def jac(x):
        return res(x), np.array([[2 * x[0]]])

    out = levenberg_marquardt(res, jac, np.array([1e-3]), max_iter=3, tol=0.0)
    lams = [h[1] for h in out.history]
    assert lams[0] == 1e-3
    assert all(b in (a * 10.0, max(a * 0.1, 1e-10)) for a, b in zip(lams, lams[1:]))


def test_clamps_and_contract_tables():
    x = clamp([-1.0, -1.0, -1.0, 2.0, -1.0])
    assert np.allclose(x, [1e-4, 1e-5, 1e-4, 0.999, 1e-6])
    s = Surface.grid(100.0, 0.02, [0.9, 1.0, 1.1], [0.5, 1.0])
    P, I = contract_tables(s, np.array([[1.0, 0.05, 0.3, -0.5, 0.04], [2.0, 0.06, 0.4, -0.6, 0.05]]))
    assert P.shape == (12, 12) and I.shape == (12, 3)
    assert np.allclose(P[:6, 8], [90, 100, 110, 90, 100, 110]) and np.allclose(P[6:, 0], 2.0)
    assert np.all(I[:, 2] == 8)


def _fake_backends(monkeypatch, A, sur_sign, centre, bias):
    """Replace the FPE and surrogate back-ends by linear models over the quotes:
    FPE prices x A^T; surrogate prices sur_sign (x - centre) A^T + centre A^T + bias."""
    from fpe_option_b200 import calibration as cal

    class FakeFpe(cal._Backend):
        def __init__(self, surface, **kw):
            super().__init__(surface)

        def steps(self, x):
            return 1e-6 * (1.0 + np.abs(x))

        def price_sets(self, xs):
            self.contracts_priced += len(xs) * len(self.surface.strikes)
            return np.atleast_2d(xs) @ A.T

    class FakeSur(cal._Backend):
        @classmethod
        def project(cls, x):
            return np.asarray(x, np.float64)

        def __init__(self, surface, pricer, grid=None):
            super().__init__(surface)
            self.fallback_quotes = 0

        def steps(self, x):
            return 1e-6 * (1.0 + np.abs(x))

        def price_sets(self, xs):
            xs = np.atleast_2d(xs)
            return (sur_sign * (xs - centre) + centre) @ A.T + bias

    monkeypatch.setattr(cal, "FpeSurface", FakeFpe)
    monkeypatch.setattr(cal, "SurrogateSurface", FakeSur)
    return cal


class _Pricer:
    last_spread = np.zeros(1)


@pytest.mark.parametrize("sur_sign,expect", [(-1.0, "hybrid->fpe"), (1.0, "hybrid")])
def test_hybrid_polish_falls_back_to_fpe_jacobians(monkeypatch, sur_sign, expect):
    """A surrogate whose Jacobian points the wrong way (reflected model) makes
    every hybrid step raise the FPE residual; the polish then finishes on FPE
    Jacobians and still reaches the FPE fit.  With a faithful Jacobian the
    hybrid polish alone gets there."""
    rng = np.random.default_rng(3)
    A = rng.standard_normal((15, 5))
    truth = np.array([1.5, 0.06, 0.4, -0.5, 0.05])
    centre = truth + np.array([0.3, 0.01, 0.05, 0.1, 0.01])
    cal = _fake_backends(monkeypatch, A, sur_sign, centre, 0.01 * rng.standard_normal(15))
    surf = cal.Surface.grid(100.0, 0.02, [0.9, 1.0, 1.1], [0.5, 1.0, 1.5, 2.0, 2.5])
    surf.prices = truth @ A.T
    x0 = truth + np.array([-0.4, 0.02, -0.1, 0.2, 0.02])
    x, info = cal.calibrate_with_surrogate(surf, _Pricer(), x0, polish="hybrid", polish_iter=10)
    assert info["polish"] == expect
    assert np.abs(x - truth).max() < 1e-6, (x, truth, info)


def test_reference_objective_backend_carries_the_reference_settings():
    """ReferenceObjectiveSurface prices with the objective's own settings
    (objective.mojo:86-104: 8 x 8 knots, num_insert 251, rtol 1e-5, atol 1e-7,
    max_step 0.02, first_step 0 = the solver's estimate, its own density sum)
    and the calibrator's FD step 1e-6 (1 + |x|) (calibrator.mojo:64-74)."""
    from fpe_option_b200.calibration import ReferenceObjectiveSurface

    surf = Surface.grid(100.0, 0.02, [0.9, 1.0, 1.1], [0.5, 1.0])
    be = ReferenceObjectiveSurface(surf)
    o = be.options
    assert be.grid == (8, 8)
    assert (o.disc, o.precision, o.num_insert, o.complex_solve, o.radau_constants) == (0, 0, 251, 1, 1)
    assert (o.rtol, o.atol, o.max_step, o.price_rule) == (1e-5, 1e-7, 0.02, 1)
    assert o.first_step < 0
    x = np.array([1.5, 0.06, 0.4, -0.5, 0.05])
    np.testing.assert_allclose(be.steps(x), 1e-6 * (1.0 + np.abs(x)))
    P, I = contract_tables(surf, x, be.grid)
    assert (I[:, :2] == 8).all() and (I[:, 2] == 8).all()


def test_interpolate_pdf_rejects_bad_shapes_before_any_device_work():
    import fpe_option_b200 as fpe

    with pytest.raises(ValueError):
        fpe.interpolate_pdf([0.0, 1.0], [0.0, 1.0, 2.0], np.zeros((2, 2)), [0.5], [0.5])
    with pytest.raises(ValueError):
        fpe.interpolate_pdf([0.0], [0.0, 1.0], np.zeros((1, 2)), [0.5], [0.5])
    with pytest.raises(ValueError):
        fpe.interpolate_pdf([0.0, 1.0], [0.0, 1.0], np.zeros((2, 2)), [0.5, 0.7], [0.5])


def test_defect_correction_reaches_the_fpe_fit(monkeypatch):
    """A surrogate that is off by a 5 % perturbation of the FPE model's linear
    map plus a bias fits the quotes to a wrong x on its own; defect correction
    (each outer iteration: one FPE pricing at the fit, then LM on the surrogate
    plus that defect) contracts the error by about the perturbation's size per
    iteration, so three iterations reach the FPE fit to ~1e-4 of the start."""
    from fpe_option_b200 import calibration as cal

    rng = np.random.default_rng(7)
    A = rng.standard_normal((15, 5))
    As = A * (1.0 + 0.05 * rng.standard_normal(A.shape))
    bias = 0.05 * rng.standard_normal(15)

    class FakeFpe(cal._Backend):
        def __init__(self, surface, **kw):
            super().__init__(surface)

        def steps(self, x):
            return 1e-6 * (1.0 + np.abs(x))

        def price_sets(self, xs):
            self.contracts_priced += len(xs) * len(self.surface.strikes)
            return np.atleast_2d(xs) @ A.T

    class FakeSur(cal._Backend):
        @classmethod
        def project(cls, x):
            return np.asarray(x, np.float64)

        def __init__(self, surface, pricer, grid=None):
            super().__init__(surface)
            self.fallback_quotes = 0

        def steps(self, x):
            return 1e-6 * (1.0 + np.abs(x))

        def price_sets(self, xs):
            return np.atleast_2d(xs) @ As.T + bias

    monkeypatch.setattr(cal, "FpeSurface", FakeFpe)
    monkeypatch.setattr(cal, "SurrogateSurface", FakeSur)
    surf = cal.Surface.grid(100.0, 0.02, [0.9, 1.0, 1.1], [0.5, 1.0, 1.5, 2.0, 2.5])
    truth = np.array([1.5, 0.06, 0.4, -0.5, 0.05])
    surf.prices = truth @ A.T
    x0 = truth + np.array([-0.4, 0.02, -0.1, 0.2, 0.02])
    # a noise level above any residual keeps the surrogate's own fit (no FPE polish)
    x_plain, _ = cal.calibrate_with_surrogate(surf, _Pricer(), x0, polish="none", quote_noise=1e6)
    x_def, info = cal.calibrate_with_surrogate(surf, _Pricer(), x0, polish="defect", defect_iter=3,
                                               defect_xtol=0.0)
    err0 = np.abs(x0 - truth).max()
    assert np.abs(x_plain - truth).max() > 1e-2 * err0  # the surrogate alone misses
    assert np.abs(x_def - truth).max() < 1e-3 * err0, (x_def, truth, info)
