"""CPU checks of the Levenberg-Marquardt restatement (reference
src/numerics/optim/lm.mojo:29-121) and the calibrator clamps
(src/engines/calibrator/calibrator.mojo:15-29)."""
import numpy as np

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
