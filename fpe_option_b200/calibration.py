"""Heston calibration by Levenberg-Marquardt on the B200 pricers.

``levenberg_marquardt`` restates the reference optimizer
(src/numerics/optim/lm.mojo:29-121): damped normal equations
(J^T J + lambda I) delta = -J^T r, lambda starting at 1e-3, x10 after a
rejected step and x0.1 (floored at 1e-10) after an accepted one, stop when
||J^T r||_inf < tol.  Parameters are (kappa, theta, sigma, rho, V0) with the
reference's clamps (src/engines/calibrator/calibrator.mojo:15-29) and a central
finite-difference Jacobian (:64-74).

Residual back-ends price the whole surface per call:

* ``FpeSurface``: the batched FPE solver.  A Jacobian is one GPU batch of
  11 x (number of quotes) contracts (the base point and ten perturbed
  parameter sets).  Its difference step is 1e-3 (1 + |x|), not the
  reference's 1e-6: an adaptive-step solver at rtol 1e-6 changes its step
  sequence between neighbouring parameter sets, which makes 1e-6 differences
  noise.
* ``ReferenceObjectiveSurface``: the reference calibrator's own objective
  (an 8 x 8 reference-discretization solve per quote and its undiscounted
  density integration) for parity with that calibrator
  (``calibrate_reference_objective``).
* ``SurrogateSurface``: the tensor-core MLP ensemble; a Jacobian costs
  microseconds.  Its step is 2 % of the parameter's training range, coarser
  than the BF16 rounding of the network's inputs.  Inside the loop quotes
  outside the training box are priced by the FPE solver; the ensemble mean
  answers the rest.

``calibrate_with_surrogate`` runs LM on the surrogate, then polishes on the
FPE solver: LM whose residuals are FPE prices of the whole surface (every
quote falls back to the solver, whatever the members' disagreement, which is
reported) and whose Jacobians are the surrogate's.  Its fixed point
J_sur^T r_FPE = 0 is the FPE least-squares fit up to a term of second order
in the Jacobian error times the residual, and each iteration costs one FPE
pricing of the surface instead of eleven.  When no hybrid step lowers the
FPE residual (the surrogate's Jacobian is no descent direction there, e.g.
at a fit pinned to the edge of its training box), FPE Jacobians finish the
polish.  ``polish="fpe"`` uses FPE Jacobians throughout; ``polish="none"`` keeps the surrogate's fit if its FPE
residual RMS is within ``noise_ratio`` times the quotes' noise level.

``polish="defect"`` corrects the surrogate instead of polishing on the FPE
solver (defect correction, also known as output space mapping): at the
current fit x_k one FPE pricing of the surface gives the surrogate's defect
d_k = p_FPE(x_k) - p_sur(x_k), and LM on the corrected surrogate
p_sur(x) + d_k - quotes gives x_{k+1}.  A fixed point satisfies
J_sur^T (p_FPE(x) - quotes) = 0, the hybrid polish's condition, while each
outer iteration costs one FPE pricing of the surface and a surrogate fit of
microsecond residuals; the defect varies slowly in x, so two or three
iterations settle it.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

PARAM_NAMES = ("kappa", "theta", "sigma", "rho", "V0")


def clamp(x: np.ndarray) -> np.ndarray:
    """Reference clamps (calibrator.mojo:15-29)."""
    x = np.array(x, dtype=np.float64)
    x[0] = max(x[0], 1e-4)
    x[1] = max(x[1], 1e-5)
    x[2] = max(x[2], 1e-4)
    x[3] = min(0.999, max(-0.999, x[3]))
    x[4] = max(x[4], 1e-6)
    return x


@dataclass
class LMResult:
    x: np.ndarray
    iterations: int
    residual_evals: int
    cost: float
    history: list = field(default_factory=list)
    stop: str = "max_iter"  # gradient, xtol, ftol, max_rejects or max_iter


def levenberg_marquardt(residual, jacobian, x0, max_iter: int = 50, tol: float = 1e-10,
                        lambda_init: float = 1e-3, lambda_up: float = 10.0,
                        lambda_down: float = 0.1, xtol: float | None = None,
                        ftol: float | None = None, max_rejects: int | None = None) -> LMResult:
    """Reference LM (lm.mojo:29-121).  jacobian(x) returns (r(x), J(x)).

    Stopping tests beyond the reference's gradient test (all off by default),
    for fits whose residual cannot reach it (quote noise, a solver's rounding
    and step-control noise): xtol stops after an accepted step with
    |delta|_inf <= xtol (|x|_inf + xtol); ftol after an accepted step that
    lowers the cost by less than ftol * cost; max_rejects after that many
    rejected steps in a row."""
    x = np.array(x0, dtype=np.float64)
    lam = lambda_init
    evals = 0
    hist = []
    it = 0
    cost = np.inf
    rejects = 0
    stop = "max_iter"
    for it in range(1, max_iter + 1):
        r, J = jacobian(x)
        evals += 1
        g = J.T @ r
        cost = float(r @ r)
        hist.append((cost, lam))
        if np.max(np.abs(g)) < tol:
            stop = "gradient"
            break
        A = J.T @ J + lam * np.eye(len(x))
        delta = np.linalg.solve(A, -g)
        x_new = x + delta
        r_new = residual(x_new)
        evals += 1
        c_new = float(r_new @ r_new)
        if c_new < cost:
            x = x_new
            lam = max(lam * lambda_down, 1e-10)
            rejects = 0
            if xtol is not None and np.max(np.abs(delta)) <= xtol * (np.max(np.abs(x)) + xtol):
                stop = "xtol"
                break
            if ftol is not None and cost - c_new < ftol * cost:
                cost = c_new
                stop = "ftol"
                break
        else:
            lam = lam * lambda_up
            rejects += 1
            if max_rejects is not None and rejects >= max_rejects:
                stop = "max_rejects"
                break
    return LMResult(x=x, iterations=it, residual_evals=evals, cost=cost, history=hist, stop=stop)


@dataclass
class Surface:
    """Quotes of one underlying: strikes and maturities (flattened), market prices."""
    S0: float
    r: float
    strikes: np.ndarray
    maturities: np.ndarray
    prices: np.ndarray
    option_type: int = 8

    @staticmethod
    def grid(S0, r, k_over_s, maturities, option_type=8):
        K, T = np.meshgrid(np.asarray(k_over_s) * S0, np.asarray(maturities), indexing="xy")
        return Surface(S0, r, K.ravel(), T.ravel(), np.zeros(K.size), option_type)


def contract_tables(surface: Surface, xs: np.ndarray, grid=(48, 24)):
    """Contract tables for every parameter vector in xs (rows) over the surface."""
    xs = np.atleast_2d(xs)
    m = len(surface.strikes)
    n = len(xs) * m
    P = np.zeros((n, 12))
    I = np.zeros((n, 3), np.int32)
    for k, x in enumerate(xs):
        x = clamp(x)
        sl = slice(k * m, (k + 1) * m)
        P[sl, 0], P[sl, 1], P[sl, 2], P[sl, 3] = x[0], x[1], x[2], x[3]
        P[sl, 4] = surface.r
        P[sl, 5] = surface.maturities
        P[sl, 6] = surface.S0
        P[sl, 7] = x[4]
        P[sl, 8] = surface.strikes
        P[sl, 11] = 3.0 * surface.S0
    I[:, 0], I[:, 1] = grid
    I[:, 2] = surface.option_type
    return P, I


class _Backend:
    """Residuals r(x) = model(x) - market over the surface, and batched central
    finite-difference Jacobians."""

    def __init__(self, surface: Surface):
        self.surface = surface
        self.contracts_priced = 0
        self.seconds = 0.0

    def price_sets(self, xs: np.ndarray) -> np.ndarray:  # (len(xs), m)
        raise NotImplementedError

    def steps(self, x: np.ndarray) -> np.ndarray:
        raise NotImplementedError

    def residual(self, x):
        return self.price_sets(np.atleast_2d(x))[0] - self.surface.prices

    def jacobian(self, x):
        """(r(x), J(x)); the pair for the last x is kept, so the repeated call
        after a rejected LM step (same x) prices nothing."""
        x = np.asarray(x, np.float64)
        if getattr(self, "_jx", None) is not None and np.array_equal(self._jx, x):
            return self._jr, self._jJ
        h = self.steps(x)
        xs = [x]
        for j in range(len(x)):
            for s in (+1.0, -1.0):
                y = x.copy()
                y[j] += s * h[j]
                xs.append(y)
        p = self.price_sets(np.array(xs))
        r = p[0] - self.surface.prices
        J = np.empty((len(r), len(x)))
        for j in range(len(x)):
            J[:, j] = (p[1 + 2 * j] - p[2 + 2 * j]) / (2.0 * h[j])
        self._jx, self._jr, self._jJ = x.copy(), r, J
        return r, J


class FpeSurface(_Backend):
    """Residuals from the batched FPE solver."""

    def __init__(self, surface: Surface, options=None, grid=(48, 24), rel_step: float = 1e-3):
        from . import BatchOptions

        super().__init__(surface)
        self.options = options or BatchOptions(disc=1, precision=1, rtol=1e-6, atol=1e-8,
                                               complex_solve=2, radau_constants=2)
        self.grid = grid
        self.rel_step = rel_step

    def steps(self, x):
        return self.rel_step * (1.0 + np.abs(x))

    def price_sets(self, xs):
        from . import price_batch

        t = time.perf_counter()
        P, I = contract_tables(self.surface, xs, self.grid)
        p, st = price_batch(P, I, self.options)
        if np.any(st != 0):
            raise RuntimeError(f"FPE pricing failed (status {sorted(set(st[st != 0].tolist()))})")
        self.contracts_priced += len(P)
        self.seconds += time.perf_counter() - t
        return p.reshape(len(xs), -1)


class ReferenceObjectiveSurface(FpeSurface):
    """Residuals of the reference calibrator's own objective
    (src/engines/calibrator/objective.mojo:66-104), priced on the GPU.

    Each quote is an FPE solve on the reference discretization with 8 x 8
    knots and the FPEDomain default of 251 grid inserts (:94), the FPESolver
    settings rtol 1e-5, atol 1e-7, max_step 0.02 and first_step 0, i.e. the
    Radau solver's own first step (:86-88), and the objective's integration of
    the terminal density: payoff max(S - K, 0) times pdf times half the
    neighbour spacing in s and v (1 at both ends), undiscounted (:26-50).  The
    FP64 factors, GMRES(10) stage solve and the reference's Radau constants
    are the reference's arithmetic.  The Jacobian step is the calibrator's
    1e-6 (1 + |x|) (calibrator.mojo:64-74).  All quotes of a residual or
    Jacobian go to the solver as one batch."""

    def __init__(self, surface: Surface, grid=(8, 8), rel_step: float = 1e-6):
        from . import BatchOptions

        opts = BatchOptions(disc=0, precision=0, num_insert=251, rtol=1e-5, atol=1e-7,
                            complex_solve=1, radau_constants=1, max_step=0.02, first_step=-1.0,
                            price_rule=1)
        super().__init__(surface, options=opts, grid=grid, rel_step=rel_step)


class SurrogateSurface(_Backend):
    """Residuals from a SurrogatePricer (FPE fall-back for untrusted quotes).
    Parameter vectors are projected into the surrogate's training box before
    pricing, so the search never leaves the region the network was fitted on."""

    # training box of (kappa, theta, sigma, rho, V0)
    LO = np.array([0.5, 0.02, 0.1, -0.9, 0.02])
    HI = np.array([3.0, 0.15, 0.8, 0.0, 0.2])
    _RANGE = HI - LO

    @classmethod
    def project(cls, x):
        return np.clip(np.asarray(x, np.float64), cls.LO, cls.HI)

    def __init__(self, surface: Surface, pricer, grid=(48, 24), frac_step: float = 0.02):
        super().__init__(surface)
        self.pricer = pricer
        self.grid = grid
        self.frac_step = frac_step
        self.fallback_quotes = 0

    def steps(self, x):
        return self.frac_step * self._RANGE

    def jacobian(self, x):
        """As the base class, with the difference stencil moved inside the box
        where x lies on or near its edge (a projected stencil would flatten
        the column)."""
        h = self.steps(x)
        c = np.clip(np.asarray(x, np.float64), self.LO + h, self.HI - h)
        r = self.residual(x)
        _, J = super().jacobian(c)
        return r, J

    def price_sets(self, xs):
        t = time.perf_counter()
        P, I = contract_tables(self.surface, np.array([self.project(x) for x in np.atleast_2d(xs)]), self.grid)
        p, fb = self.pricer.price(P, I, gate_disagreement=False)
        self.fallback_quotes += int(fb.sum())
        self.contracts_priced += int(fb.sum())  # FPE solves spent inside the loop
        self.seconds += time.perf_counter() - t
        return p.reshape(len(xs), -1)


STOP = {"xtol": 1e-6, "ftol": 1e-4, "max_rejects": 6}


class HybridSurface:
    """FPE residuals with the surrogate's Jacobians (see the module notes)."""

    def __init__(self, fpe: FpeSurface, sur: SurrogateSurface):
        self.fpe, self.sur = fpe, sur

    def residual(self, x):
        return self.fpe.residual(x)

    def jacobian(self, x):
        _, J = self.sur.jacobian(x)
        return self.fpe.residual(x), J


class DefectSurface:
    """The surrogate's residual plus a fixed defect vector (FPE minus surrogate
    prices at the last outer iterate)."""

    def __init__(self, sur: SurrogateSurface, defect: np.ndarray):
        self.sur, self.defect = sur, defect

    def residual(self, x):
        return self.sur.residual(x) + self.defect

    def jacobian(self, x):
        r, J = self.sur.jacobian(x)
        return r + self.defect, J


def calibrate_reference_objective(surface: Surface, x0, max_iter=50, tol=1e-8, **kw):
    """The reference Calibrator (calibrator.mojo:87-119): LM with lambda 1e-3,
    x10 / x0.1 (lm.mojo:29-121) on the reference objective, the parameters
    clamped as in _vec_to_params.  Only call quotes (option type 8) exist in
    that objective.  Returns (x, info)."""
    be = ReferenceObjectiveSurface(surface, **kw)
    t = time.perf_counter()
    res = levenberg_marquardt(be.residual, be.jacobian, x0, max_iter=max_iter, tol=tol)
    return clamp(res.x), {"seconds": time.perf_counter() - t, "fpe_contracts": be.contracts_priced,
                          "iterations": res.iterations, "cost": res.cost, "stop": res.stop}


def calibrate_fpe(surface: Surface, x0, max_iter=40, tol=1e-10, **kw):
    be = FpeSurface(surface, **kw)
    t = time.perf_counter()
    res = levenberg_marquardt(be.residual, be.jacobian, x0, max_iter=max_iter, tol=tol, **STOP)
    return clamp(res.x), {"seconds": time.perf_counter() - t, "fpe_contracts": be.contracts_priced,
                          "iterations": res.iterations, "cost": res.cost}


def calibrate_with_surrogate(surface: Surface, pricer, x0, max_iter=50, tol=1e-10,
                             polish: str = "hybrid", quote_noise: float | None = None,
                             noise_ratio: float = 1.5, polish_iter: int = 10, fpe_kw=None,
                             defect_iter: int = 3, defect_xtol: float = 1e-4):
    """Surrogate-in-loop LM, FPE verification, optional FPE polish or defect
    correction (see the module notes)."""
    fpe_kw = fpe_kw or {}
    t = time.perf_counter()
    sb = SurrogateSurface(surface, pricer, grid=fpe_kw.get("grid", (48, 24)))
    res = levenberg_marquardt(sb.residual, sb.jacobian, SurrogateSurface.project(x0), max_iter=max_iter,
                              tol=tol, xtol=1e-5, ftol=1e-6, max_rejects=6)
    x = clamp(SurrogateSurface.project(res.x))
    x_sur = x.copy()
    fb = FpeSurface(surface, **fpe_kw)
    r_fpe = fb.residual(x)
    r_sur = sb.residual(x)
    spread = float(np.max(pricer.last_spread))
    rms_fpe = float(np.sqrt(np.mean(r_fpe ** 2)))
    polished = False
    it_polish = 0
    polish_used = polish
    if polish == "defect":
        # r_fpe = p_FPE(x) - quotes, r_sur = p_sur(x) - quotes: their difference is the defect
        for _ in range(defect_iter):
            d = r_fpe - r_sur
            db = DefectSurface(sb, d)
            cor = levenberg_marquardt(db.residual, db.jacobian, x, max_iter=max_iter, tol=tol, xtol=1e-5,
                                      ftol=1e-6, max_rejects=6)
            x_new = clamp(SurrogateSurface.project(cor.x))
            it_polish += 1
            step = float(np.max(np.abs(x_new - x) / np.maximum(np.abs(x), 1e-8)))
            x = x_new
            r_fpe = fb.residual(x)
            r_sur = sb.residual(x)
            if step < defect_xtol:
                break
        polished = True
    elif polish == "hybrid":
        hb = HybridSurface(fb, sb)
        # near-Gauss-Newton steps: the fit starts close to the optimum
        pol = levenberg_marquardt(hb.residual, hb.jacobian, x, max_iter=polish_iter, tol=tol,
                                  lambda_init=1e-9, **STOP)
        it_polish = pol.iterations
        if np.array_equal(pol.x, x) and pol.stop != "gradient":
            # no step was accepted: the surrogate's Jacobian gives no descent
            # direction for the FPE residual here, so the FPE's own finishes
            polish_used = "hybrid->fpe"
            pol = levenberg_marquardt(fb.residual, fb.jacobian, x, max_iter=polish_iter, tol=tol, **STOP)
            it_polish += pol.iterations
        x = clamp(pol.x)
        polished = True
    elif polish == "fpe" or (polish == "none" and (quote_noise is None or rms_fpe > noise_ratio * quote_noise)):
        pol = levenberg_marquardt(fb.residual, fb.jacobian, x, max_iter=polish_iter, tol=tol, **STOP)
        x = clamp(pol.x)
        polished = True
        it_polish = pol.iterations
    return x, {"seconds": time.perf_counter() - t,
               "fpe_contracts": fb.contracts_priced + sb.contracts_priced,
               "surrogate_iterations": res.iterations, "polished": polished, "polish": polish_used,
               "polish_iterations": it_polish, "fallback_quotes": sb.fallback_quotes,
               "max_disagreement_at_fit": spread, "x_surrogate_fit": x_sur.tolist(),
               "fpe_rms_at_surrogate_fit": rms_fpe,
               "surrogate_rms_at_fit": float(np.sqrt(np.mean(r_sur ** 2)))}
