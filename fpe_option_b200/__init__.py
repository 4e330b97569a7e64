"""B200-native Heston Fokker-Planck option pricing.

Drop-in for the reference Python API (elevenwang-creator/FPE_option,
python/fpe_engine/__init__.py and pricer.py): ``price()`` (one-shot with
Greeks), ``Compute`` (stepwise, lazily cached intermediates), the result
dataclasses and ``FpeParams``.  Everything computes on the GPU through the C
ABI of ``libfpe_engine.so``; there is no CPU fallback.

Additions: ``price_batch`` / ``Plan`` price thousands of contracts with
different parameters, barriers and grid sizes in one launch sequence;
``heston_cf_price`` prices Europeans from the Heston characteristic function.

Usage::

    import fpe_option_b200 as fpe
    r = fpe.price(S0=60.0, K=[80.0, 90.0], s_max=150.0)
    c = fpe.Compute(S0=60.0, V0=0.1, T=0.6, r=0.1)
    c.payoff_price([100.0])
"""
from __future__ import annotations

import ctypes as C
import logging
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib

__version__ = "0.1.0"
_logger = logging.getLogger("fpe_engine")

__all__ = [
    "price", "Compute", "FpeParams", "PriceResult", "KnotsResult", "GridPointsResult",
    "Basis1DResult", "GreeksResult", "is_available", "price_batch", "Plan", "Contract",
    "BatchOptions", "OPTION_TYPES", "heston_cf_price", "interpolate_pdf",
]

# python/fpe_engine/__init__.py:54-60
OPTION_TYPES = {
    "down_and_in_call": 0, "down_and_in_put": 1,
    "down_and_out_call": 2, "down_and_out_put": 3,
    "up_and_in_call": 4, "up_and_in_put": 5,
    "up_and_out_call": 6, "up_and_out_put": 7,
    "european_call": 8, "european_put": 9,
}
_OPTION_TYPES = OPTION_TYPES
MAX_STRIKES = 1024  # src/bindings/_params.mojo:5


@dataclass
class PriceResult:  # python/fpe_engine/pricer.py:13-18
    prices: np.ndarray
    deltas: np.ndarray
    gammas: np.ndarray
    vegas: np.ndarray


@dataclass
class KnotsResult:  # pricer.py:21-24
    s: np.ndarray
    v: np.ndarray


@dataclass
class GridPointsResult:  # pricer.py:27-32
    s: np.ndarray
    v: np.ndarray
    s_weights: np.ndarray
    v_weights: np.ndarray


@dataclass
class Basis1DResult:  # pricer.py:35-40
    Bs: object
    dBs: object
    Bv: object
    dBv: object


@dataclass
class GreeksResult:  # pricer.py:43-47
    delta: np.ndarray
    gamma: np.ndarray
    vega: np.ndarray


@dataclass
class FpeParams:  # pricer.py:66-94
    kappa: float = 1.2
    theta: float = 0.05
    sigma: float = 0.35
    rho: float = -0.4
    r: float = 0.05
    T: float = 0.5
    S0: float = 100.0
    V0: float = 0.1
    n_s: int = 38
    n_v: int = 38
    option_type: str | int = "european_call"
    K: float | list | None = None
    barrier: float = 0.0
    s_min: float | None = None
    s_max: float | None = None

    def __post_init__(self):
        if isinstance(self.option_type, str):
            if self.option_type not in _OPTION_TYPES:
                raise ValueError(f"unknown option_type '{self.option_type}'")
        else:
            if not (0 <= self.option_type <= 9):
                raise ValueError(f"option_type must be 0-9, got {self.option_type}")
        if not (4 <= self.n_s <= 256):
            raise ValueError(f"n_s must be in [4, 256], got {self.n_s}")
        if not (4 <= self.n_v <= 256):
            raise ValueError(f"n_v must be in [4, 256], got {self.n_v}")


def is_available() -> bool:
    """True when the CUDA library is built and a GPU can run it."""
    try:
        return bool(_lib.load().fpe_device_available())
    except Exception as e:  # the library is missing or CUDA is unusable
        _logger.warning("FPE GPU engine not available: %s", e)
        return False


def _require():
    L = _lib.load()
    if not L.fpe_device_available():
        raise RuntimeError("FPE GPU engine not available (no usable CUDA device)")
    from . import autotune

    autotune.load_default()  # the tuned solve shapes measured on a B200, once
    return L


def _option_type_int(ot) -> int:
    if isinstance(ot, str):
        if ot not in _OPTION_TYPES:
            raise ValueError(f"unknown option_type '{ot}'")
        return _OPTION_TYPES[ot]
    if isinstance(ot, (bool,)) or not isinstance(ot, (int, np.integer)):
        raise ValueError("option_type must be str or int")
    v = int(ot)
    if v < 0 or v > 9:
        raise ValueError(f"option_type must be 0-9, got {v}")
    return v


def _strikes(K) -> list[float]:
    if isinstance(K, np.ndarray):
        K = K.tolist()
    if isinstance(K, (int, float, np.floating, np.integer)) and not isinstance(K, bool):
        return [float(K)]
    if isinstance(K, (list, tuple)):
        if len(K) > MAX_STRIKES:
            raise ValueError(f"K list too large, max {MAX_STRIKES}")
        return [float(k) for k in K]
    raise ValueError("K must be float, int, or list of floats")


def _validate(kappa, theta, sigma, rho, r, T, S0, V0, n_s, n_v, barrier, ot, s_min, s_max, K):
    """fpe_params_from_kwargs (src/bindings/_params.mojo:53-121)."""
    if n_s < 4 or n_s > 256:
        raise ValueError(f"n_s must be in [4, 256], got {n_s}")
    if n_v < 4 or n_v > 256:
        raise ValueError(f"n_v must be in [4, 256], got {n_v}")
    if len(K) == 0:
        raise ValueError("K must not be empty")
    ok = (kappa > 0 and theta > 0 and sigma > 0 and T > 0 and S0 > 0 and V0 >= 0 and s_min >= 0
          and s_max > s_min and -1 <= rho <= 1)
    if not ok:
        raise ValueError("invalid Heston parameters")
    valid = all(k > 0 for k in K)
    if ot <= 3:
        valid &= 0 < barrier < S0
    elif ot <= 7:
        valid &= barrier > 0 and barrier >= S0
    else:
        valid &= barrier == 0.0
    if not valid:
        raise ValueError("invalid FPE parameters (check barrier/option_type combo)")


def _arr(ptr, n) -> np.ndarray:
    if n <= 0 or not ptr:
        return np.zeros(0, dtype=np.float64)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(np.float64, copy=True)


def price(
    kappa: float = 1.2, theta: float = 0.05, sigma: float = 0.35,
    rho: float = -0.4, r: float = 0.1, T: float = 0.6,
    S0: float = 60.0, V0: float = 0.1,
    K: list[float] | float = 100.0, barrier: float = 0.0,
    option_type: str | int = "european_call",
    n_s: int = 38, n_v: int = 38,
    s_min: float | None = None, s_max: float | None = None,
) -> PriceResult:
    """One-shot price + Greeks (python/fpe_engine/__init__.py:63-103).

    Runs the base pricing and the four bumped pricings of the reference
    PricingEngine (num_insert 50, rtol 1e-4, atol 1e-6) as one GPU batch.
    """
    try:
        L = _require()
    except RuntimeError:
        raise
    except Exception as e:
        raise RuntimeError(f"FPE GPU engine not available: {e}") from e
    Ks = _strikes(K)
    ot = _option_type_int(option_type)
    smin = 0.0 if s_min is None else float(s_min)
    smax = S0 * 3.0 if s_max is None else float(s_max)
    _validate(kappa, theta, sigma, rho, r, T, S0, V0, n_s, n_v, barrier, ot, smin, smax, Ks)
    k = np.ascontiguousarray(Ks, dtype=np.float64)
    res = _lib.FpeOneshotResult()
    L.fpe_price_oneshot(kappa, theta, sigma, rho, r, T, S0, V0,
                        k.ctypes.data_as(_lib.dp), len(k), barrier, ot, n_s, n_v, 50,
                        smin, smax, C.byref(res))
    if res.len != len(k):
        raise RuntimeError("FPE GPU pricing failed")
    try:
        return PriceResult(prices=_arr(res.price, res.len), deltas=_arr(res.delta, res.len),
                           gammas=_arr(res.gamma, res.len), vegas=_arr(res.vega, res.len))
    finally:
        L.fpe_compute_free_oneshot(C.byref(res))


def _csr(L, handle, which):
    import scipy.sparse as sp
    nr, nc = C.c_int32(), C.c_int32()
    nnz = L.fpe_compute_basis_csr(handle, which, C.byref(nr), C.byref(nc), None, None, None)
    if nnz < 0:
        raise RuntimeError("basis export failed")
    indptr = np.empty(nr.value + 1, np.int32)
    indices = np.empty(nnz, np.int32)
    data = np.empty(nnz, np.float64)
    L.fpe_compute_basis_csr(handle, which, C.byref(nr), C.byref(nc),
                            indptr.ctypes.data_as(_lib.ip), indices.ctypes.data_as(_lib.ip),
                            data.ctypes.data_as(_lib.dp))
    return sp.csr_matrix((data, indices, indptr), shape=(nr.value, nc.value))


class Compute:
    """Stepwise FPE computation context (python/fpe_engine/pricer.py:104-197).

    Construction builds the domain, quadrature, basis and Galerkin factors on
    the GPU eagerly; the initial condition, the solve and the PDF are computed
    on first access and cached (Python side: repeated access returns the same
    object).  Keyword defaults follow src/bindings/_params.mojo:53-71 and
    _py_pipeline.mojo:24 (num_insert 251).
    """

    def __init__(self, **kwargs):
        if "option_type" not in kwargs:
            kwargs["option_type"] = "european_put"
        kw = {k: v for k, v in kwargs.items() if v is not None}
        L = _require()
        g = kw.get
        self.kappa, self.theta = float(g("kappa", 1.2)), float(g("theta", 0.05))
        self.sigma, self.rho = float(g("sigma", 0.35)), float(g("rho", -0.4))
        self.r, self.T = float(g("r", 0.05)), float(g("T", 0.5))
        self.S0, self.V0 = float(g("S0", 100.0)), float(g("V0", 0.1))
        self.n_s, self.n_v = int(g("n_s", 38)), int(g("n_v", 38))
        self.barrier = float(g("barrier", 0.0))
        self.s_min = float(g("s_min", 0.0))
        self.s_max = float(g("s_max", self.S0 * 3.0))
        self.num_insert = int(g("num_insert", 251))
        self.option_type = _option_type_int(kw["option_type"])
        Ks = _strikes(kw["K"]) if "K" in kw else [100.0]
        _validate(self.kappa, self.theta, self.sigma, self.rho, self.r, self.T, self.S0, self.V0,
                  self.n_s, self.n_v, self.barrier, self.option_type, self.s_min, self.s_max, Ks)
        opt = _lib.FpeBatchOptions()
        opt.num_insert = self.num_insert
        opt.disc = int(g("disc", 0))
        opt.precision = int(g("precision", 0))
        self._L = L
        self._h = L.fpe_compute_create_ex(self.kappa, self.theta, self.sigma, self.rho, self.r,
                                          self.T, self.S0, self.V0, self.n_s, self.n_v,
                                          self.barrier, self.option_type, self.s_min, self.s_max,
                                          C.byref(opt))
        if not self._h:
            raise RuntimeError("FPE GPU pipeline creation failed")
        self._knots_cache = None
        self._grid_points_cache = None
        self._basis_1d_cache = None
        self._basis_2d_cache = None
        self._ic_cache = None
        self._solve_cache = None
        self._pdf_cache = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.fpe_compute_destroy(h)
            self._h = None

    @property
    def knots(self) -> KnotsResult:
        if self._knots_cache is None:
            r = _lib.FpeVec2Result()
            self._L.fpe_compute_knots(self._h, C.byref(r))
            try:
                self._knots_cache = KnotsResult(s=_arr(r.s_data, r.s_len), v=_arr(r.v_data, r.v_len))
            finally:
                self._L.fpe_compute_free_vec2(C.byref(r))
        return self._knots_cache

    @property
    def grid_points(self) -> GridPointsResult:
        if self._grid_points_cache is None:
            r = _lib.FpeGridPtsResult()
            self._L.fpe_compute_grid_points(self._h, C.byref(r))
            try:
                self._grid_points_cache = GridPointsResult(
                    s=_arr(r.s_data, r.s_len), v=_arr(r.v_data, r.v_len),
                    s_weights=_arr(r.sw_data, r.s_len), v_weights=_arr(r.vw_data, r.v_len))
            finally:
                self._L.fpe_compute_free_grid_pts(C.byref(r))
        return self._grid_points_cache

    @property
    def basis_1d(self) -> Basis1DResult:
        if self._basis_1d_cache is None:
            self._basis_1d_cache = Basis1DResult(
                Bs=_csr(self._L, self._h, 0), dBs=_csr(self._L, self._h, 1),
                Bv=_csr(self._L, self._h, 2), dBv=_csr(self._L, self._h, 3))
        return self._basis_1d_cache

    @property
    def basis_2d(self):
        """kron(Bs, Bv) as scipy CSR (compute_pipeline.mojo:73-74)."""
        if self._basis_2d_cache is None:
            import scipy.sparse as sp
            b = self.basis_1d
            self._basis_2d_cache = sp.kron(b.Bs, b.Bv, format="csr")
        return self._basis_2d_cache

    @property
    def initial_condition(self) -> np.ndarray:
        if self._ic_cache is None:
            r = _lib.FpeVecResult()
            self._L.fpe_compute_initial_condition(self._h, C.byref(r))
            try:
                if r.len <= 0:
                    raise RuntimeError("initial condition failed")
                self._ic_cache = _arr(r.data, r.len)
            finally:
                self._L.fpe_compute_free_vec(C.byref(r))
        return self._ic_cache

    @property
    def solve(self) -> list[np.ndarray]:
        if self._solve_cache is None:
            r = _lib.FpeMatResult()
            self._L.fpe_compute_solve(self._h, C.byref(r))
            try:
                if r.n_rows <= 0:
                    raise RuntimeError("solve failed")
                m = _arr(r.data, r.n_rows * r.n_cols).reshape(r.n_rows, r.n_cols)
                self._solve_cache = [m[i].copy() for i in range(r.n_rows)]
            finally:
                self._L.fpe_compute_free_mat(C.byref(r))
        return self._solve_cache

    @property
    def pdf(self) -> np.ndarray:
        if self._pdf_cache is None:
            r = _lib.FpeMatResult()
            self._L.fpe_compute_pdf(self._h, C.byref(r))
            try:
                if r.n_rows <= 0:
                    raise RuntimeError("pdf failed")
                self._pdf_cache = _arr(r.data, r.n_rows * r.n_cols).reshape(r.n_rows, r.n_cols)
            finally:
                self._L.fpe_compute_free_mat(C.byref(r))
        return self._pdf_cache

    def pdf_interpolate(self, s, v) -> np.ndarray:
        """The terminal density at points (s, v), interpolated from the pdf grid
        (Catmull-Rom bicubic; reference src/server/interpolator.mojo)."""
        g = self.grid_points
        return interpolate_pdf(g.s, g.v, self.pdf, s, v)

    def payoff_price(self, K) -> np.ndarray:
        k = np.ascontiguousarray(_strikes(K), dtype=np.float64)
        r = _lib.FpeVecResult()
        self._L.fpe_compute_price(self._h, k.ctypes.data_as(_lib.dp), len(k), C.byref(r))
        try:
            if r.len != len(k):
                raise RuntimeError("payoff pricing failed")
            return _arr(r.data, r.len)
        finally:
            self._L.fpe_compute_free_vec(C.byref(r))

    def greeks(self, K) -> GreeksResult:
        k = np.ascontiguousarray(_strikes(K), dtype=np.float64)
        r = _lib.FpeGreeksResult()
        self._L.fpe_compute_greeks(self._h, k.ctypes.data_as(_lib.dp), len(k), 0.0, 0.0, C.byref(r))
        try:
            if r.len != len(k):
                raise RuntimeError("greeks failed")
            return GreeksResult(delta=_arr(r.delta, r.len), gamma=_arr(r.gamma, r.len),
                                vega=_arr(r.vega, r.len))
        finally:
            self._L.fpe_compute_free_greeks(C.byref(r))


# ---------------------------------------------------------------------------
# Batched API (no reference counterpart: the reference prices one contract per call)
# ---------------------------------------------------------------------------
@dataclass
class Contract:
    kappa: float
    theta: float
    sigma: float
    rho: float
    r: float
    T: float
    S0: float
    V0: float
    K: Sequence[float] | float
    option_type: int | str = 8
    barrier: float = 0.0
    n_s: int = 38
    n_v: int = 38
    s_min: float = 0.0
    s_max: float = -1.0


@dataclass
class BatchOptions:
    disc: int = 0            # 0 reference discretization, 1 config discretization
    precision: int = 0       # 0 FP64 factors, 1 FP32 factors + FP64 refinement
    num_insert: int = 50
    refine: int = 0          # extra FP64 refinement sweeps per stage solve
    complex_solve: int = 0   # 0 auto, 1 GMRES(10) (reference algorithm), 2 direct complex LU
    radau_constants: int = 0  # 0 auto, 1 the reference's U1/ALPH/BETA/TI13, 2 exact Radau IIA
    rtol: float = 1e-4
    atol: float = 1e-6
    ic_sigma_s: float = 0.6
    ic_sigma_v: float = 0.004
    ic_sub: int = 8
    greeks: bool = False
    rel_s: float = 0.01
    rel_v: float = 0.1
    max_step: float = 0.0    # <= 0: T/5 (the reference Pricer); > 0: absolute cap
    first_step: float = 0.0  # 0: 1e-6 (Pricer); < 0: the Radau solver's own estimate
    price_rule: int = 0      # 1: the calibration objective's undiscounted sum (reference disc)
    max_steps: int = 0       # <= 0: 100000 accepted steps (the reference cap)
    fp64_retry: int = 0      # precision 1: re-solve failed solves with FP64 factors (0/1 on, < 0 off)
    stage_wait_cycles: int = 0  # <= 0: ~1 s bounded wait per staged sweep stage
    block_split: int = 0     # stage-LU blocks: 0 auto, 1 nv x nv, 2 (nv/2) x (nv/2)
    sweep_buffers: int = 0   # staged-sweep buffers: 0 auto, 2..4
    knock_in_tol_scale: float = 0.0  # knock-in solve pairs: rtol/atol factor (<= 0: 1 disc 0, 0.01 disc 1)

    def to_c(self) -> _lib.FpeBatchOptions:
        o = _lib.FpeBatchOptions()
        o.disc, o.precision, o.num_insert, o.refine = (self.disc, self.precision,
                                                       self.num_insert, self.refine)
        o.rtol, o.atol = self.rtol, self.atol
        o.ic_sigma_s, o.ic_sigma_v, o.ic_sub = self.ic_sigma_s, self.ic_sigma_v, self.ic_sub
        o.greeks = 1 if self.greeks else 0
        o.rel_s, o.rel_v = self.rel_s, self.rel_v
        o.complex_solve = self.complex_solve
        o.radau_constants = self.radau_constants
        o.max_step, o.first_step, o.price_rule = self.max_step, self.first_step, self.price_rule
        o.max_steps, o.fp64_retry = self.max_steps, self.fp64_retry
        o.stage_wait_cycles = self.stage_wait_cycles
        o.block_split, o.sweep_buffers = self.block_split, self.sweep_buffers
        o.knock_in_tol_scale = self.knock_in_tol_scale
        return o


def contracts_from_arrays(params: np.ndarray, ints: np.ndarray):
    """Pack a (n, 12) parameter table [kappa theta sigma rho r T S0 V0 K barrier
    s_min s_max] and a (n, 3) int table [n_s n_v option_type] into C contracts
    (one strike each).  Returns the ctypes array and the strike buffer that
    must stay alive while it is used."""
    params = np.ascontiguousarray(params, np.float64)
    ints = np.ascontiguousarray(ints, np.int32)
    n = len(params)
    strikes = np.ascontiguousarray(params[:, 8])
    arr = (_lib.FpeContract * n)()
    base = strikes.ctypes.data
    for i in range(n):
        p, q = params[i], ints[i]
        arr[i] = _lib.FpeContract(p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[9], p[10],
                                  p[11], int(q[0]), int(q[1]), int(q[2]), 1,
                                  C.cast(base + 8 * i, _lib.dp))
    return arr, strikes


class Plan:
    """A batch resident on the device: ``run()`` enqueues the five kernel
    launches on a CUDA stream, ``results()`` waits and returns the prices."""

    def __init__(self, contracts, options: BatchOptions | None = None, _keep=None):
        L = _require()
        self._L = L
        self._keep = _keep
        self.options = options or BatchOptions()
        self._opt = self.options.to_c()
        self._c = contracts
        self._h = L.fpe_plan_create(contracts, len(contracts), C.byref(self._opt))
        if not self._h:
            raise RuntimeError("fpe_plan_create failed")
        nr, ns = C.c_int32(), C.c_int32()
        L.fpe_plan_sizes(self._h, C.byref(nr), C.byref(ns))
        self.n_results, self.n_solves = nr.value, ns.value

    def run(self, stream: int | None = None) -> int:
        n = self._L.fpe_plan_run(self._h, C.c_void_p(stream) if stream else None)
        if n < 0:
            raise RuntimeError("fpe_plan_run failed")
        return n

    def results(self):
        n = self.n_results
        p, dl, g, v = (np.zeros(n) for _ in range(4))
        st = np.zeros(n, np.int32)
        self._L.fpe_plan_results(self._h, p.ctypes.data_as(_lib.dp), dl.ctypes.data_as(_lib.dp),
                                 g.ctypes.data_as(_lib.dp), v.ctypes.data_as(_lib.dp),
                                 st.ctypes.data_as(_lib.ip))
        return p, dl, g, v, st

    def stats(self) -> dict:
        out = (C.c_int64 * 20)()
        self._L.fpe_plan_stats(self._h, out)
        keys = ["solves", "accepted", "rejected", "newton", "gmres", "lu", "admm",
                "max_ndof_s", "max_ndof_v", "total_dofs", "passes_real", "passes_complex",
                "factor_bytes", "worst_status", "kcyc_factor", "kcyc_solve", "kcyc_kron",
                "kcyc_total", "kcyc_factor_gj", "kcyc_factor_gemm"]
        return dict(zip(keys, list(out)))

    def retried(self) -> int:
        """Solves of the last ``results()`` re-solved with FP64 factors after a
        mixed-precision failure."""
        return int(self._L.fpe_plan_retried(self._h))

    def solve_info(self) -> np.ndarray:
        """Per-solve counters of the last run, (n_solves, 40) int32 in the plan's
        solve order (see fpe_plan_solve_info in include/fpe_engine.h)."""
        out = np.zeros((self.n_solves, 40), np.int32)
        if self._L.fpe_plan_solve_info(self._h, out.ctypes.data_as(_lib.ip)) < 0:
            raise RuntimeError("fpe_plan_solve_info failed")
        return out

    def kernel_times(self, stream: int | None = None) -> list[float]:
        """Run once with CUDA events around each kernel; returns ms for
        [setup, galerkin, ic, radau, payoff]."""
        ms = (C.c_float * 5)()
        if self._L.fpe_plan_kernel_times(self._h, C.c_void_p(stream) if stream else None, ms) < 0:
            raise RuntimeError("fpe_plan_kernel_times failed")
        return list(ms)

    def close(self):
        if getattr(self, "_h", None):
            self._L.fpe_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def price_batch(params: np.ndarray, ints: np.ndarray, options: BatchOptions | None = None,
                chunk: int = 8192):
    """Price n single-strike contracts; returns (prices, status).

    Batches larger than ``chunk`` contracts run as consecutive plans of at most
    ``chunk`` (a plan's device arenas grow with its solves: about 3 MB per
    solve on a 48 x 24 grid, so 8192 contracts stay near 25 GB)."""
    params = np.asarray(params)
    ints = np.asarray(ints)
    n = len(params)
    out_p = np.zeros(n)
    out_s = np.zeros(n, np.int32)
    for a in range(0, n, max(1, chunk)):
        b = min(n, a + chunk)
        arr, keep = contracts_from_arrays(params[a:b], ints[a:b])
        plan = Plan(arr, options, _keep=keep)
        try:
            plan.run()
            p, _, _, _, st = plan.results()
            out_p[a:b], out_s[a:b] = p, st
        finally:
            plan.close()
    return out_p, out_s


def heston_cf_price(params: np.ndarray, ints: np.ndarray):
    """European prices from the Heston characteristic function, FP64 on the GPU.

    Same tables as :func:`price_batch` (grid columns are ignored); rows whose
    option type is not 8 (call) or 9 (put) get NaN and status
    ``FPE_STATUS_UNSUPPORTED`` (2).  Returns (prices, status).  No reference
    counterpart: it measures the discretization error of the FPE prices."""
    _require()
    params = np.asarray(params)
    ints = np.asarray(ints)
    n = len(params)
    prices = np.zeros(n)
    status = np.zeros(n, np.int32)
    if n == 0:
        return prices, status
    arr, keep = contracts_from_arrays(params, ints)
    rc = _lib.load().fpe_heston_cf_price(arr, n, prices.ctypes.data_as(_lib.dp),
                                         status.ctypes.data_as(_lib.ip))
    del keep
    if rc < 0:
        raise RuntimeError("fpe_heston_cf_price failed")
    return prices, status


def interpolate_pdf(s_points, v_points, pdf, s, v) -> np.ndarray:
    """A density tabulated on the grid s_points x v_points (row-major pdf, e.g.
    ``Compute.pdf`` on ``Compute.grid_points``) interpolated at the points
    (s, v) on the GPU: Catmull-Rom bicubic, bilinear for grids with fewer than
    4 points per axis (reference src/server/interpolator.mojo:62-198)."""
    sp = np.ascontiguousarray(s_points, np.float64)
    vp = np.ascontiguousarray(v_points, np.float64)
    f = np.ascontiguousarray(pdf, np.float64)
    sq = np.ascontiguousarray(np.atleast_1d(s), np.float64)
    vq = np.ascontiguousarray(np.atleast_1d(v), np.float64)
    if sp.ndim != 1 or vp.ndim != 1 or len(sp) < 2 or len(vp) < 2:
        raise ValueError("interpolate_pdf: each grid axis needs at least 2 points")
    if f.shape != (len(sp), len(vp)) or sq.shape != vq.shape or sq.ndim != 1:
        raise ValueError("interpolate_pdf: pdf must be len(s_points) x len(v_points), s and v of equal length")
    L = _require()
    import torch

    n = len(sq)
    if n == 0:
        return np.zeros(0)
    dev = torch.device("cuda")
    t = [torch.from_numpy(a).to(dev) for a in (sp, vp, f, sq, vq)]
    out = torch.empty(n, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream or 1  # 1: the legacy default stream
    rc = L.fpe_pdf_interpolate(t[0].data_ptr(), len(sp), t[1].data_ptr(), len(vp), t[2].data_ptr(),
                               t[3].data_ptr(), t[4].data_ptr(), n, out.data_ptr(), stream)
    if rc != 0:
        raise RuntimeError("fpe_pdf_interpolate failed")
    return out.cpu().numpy()
