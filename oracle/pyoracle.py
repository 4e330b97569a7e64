"""ctypes binding of the CPU FP64 oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
import this module; the product package never does.  The oracle restates the
reference Mojo engine (elevenwang-creator/FPE_option); see fpe_oracle.cpp for
the file:line citations of every stage.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_fpe.so")
_lib = None


class OrcOptions(C.Structure):
    _fields_ = [
        ("disc", C.c_int32),
        ("num_insert", C.c_int32),
        ("rtol", C.c_double),
        ("atol", C.c_double),
        ("ic_sigma_s", C.c_double),
        ("ic_sigma_v", C.c_double),
        ("nnls_exact", C.c_int32),
        ("ic_sub", C.c_int32),
        ("complex_direct", C.c_int32),
        ("radau_constants", C.c_int32),
        ("max_step", C.c_double),
        ("first_step", C.c_double),
        ("price_rule", C.c_int32),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (in place, next to the sources)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        d, i32, i64, vp = C.c_double, C.c_int32, C.c_int64, C.c_void_p
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int32)
        op = C.POINTER(OrcOptions)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [d] * 8 + [i32, i32, d, i32, d, d, op]
        L.orc_destroy.argtypes = [vp]
        L.orc_len.restype = i64
        L.orc_len.argtypes = [vp, i32]
        L.orc_fill.restype = i64
        L.orc_fill.argtypes = [vp, i32, dp]
        L.orc_dims.argtypes = [vp, C.POINTER(C.c_int64)]
        L.orc_basis_csr.restype = i64
        L.orc_basis_csr.argtypes = [vp, i32, ip, ip, ip, ip, dp]
        L.orc_factor.restype = i32
        L.orc_factor.argtypes = [vp, i32, dp]
        L.orc_price_at.restype = i32
        L.orc_price_at.argtypes = [vp, dp, i32, dp]
        L.orc_greeks.restype = i32
        L.orc_greeks.argtypes = [vp, dp, i32, d, d, dp, dp, dp]
        L.orc_pricer_price.restype = i32
        L.orc_pricer_price.argtypes = [d] * 8 + [i32, i32, d, i32, d, d, dp, i32, op, dp]
        L.orc_engine_price.restype = i32
        L.orc_engine_price.argtypes = [d] * 8 + [i32, i32, d, i32, d, d, dp, i32, op, dp, dp, dp, dp]
        L.orc_price_batch.restype = i32
        L.orc_price_batch.argtypes = [i32, dp, ip, op, i32, dp]
        L.orc_pdf_interpolate.restype = C.c_int32
        L.orc_pdf_interpolate.argtypes = [dp, C.c_int32, dp, C.c_int32, dp, dp, dp, C.c_int32, dp]
        L.orc_heston_cf_price.restype = d
        L.orc_heston_cf_price.argtypes = [d] * 9 + [i32]
        L.orc_bspline_value.restype = d
        L.orc_bspline_value.argtypes = [dp, i32, i32, d, i32]
        L.orc_generate_knots.restype = i32
        L.orc_generate_knots.argtypes = [i32, i32, i32, d, d, d, d, d, dp]
        L.orc_payoff.restype = i32
        L.orc_payoff.argtypes = [i32, dp, i32, d, d, dp]
        L.orc_radau_dense.restype = i32
        L.orc_radau_dense.argtypes = [i32, dp, dp, dp, d, d, d, d, d, i32, dp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def options(disc=0, num_insert=0, rtol=0.0, atol=0.0, ic_sigma_s=0.0, ic_sigma_v=0.0,
            nnls_exact=0, ic_sub=0, complex_direct=0, radau_constants=0, max_step=0.0,
            first_step=0.0, price_rule=0) -> OrcOptions:
    return OrcOptions(disc, num_insert, rtol, atol, ic_sigma_s, ic_sigma_v, nnls_exact, ic_sub,
                      complex_direct, radau_constants, max_step, first_step, price_rule)


_ARRAYS = {"s_knots": 0, "v_knots": 1, "s": 2, "v": 3, "s_weights": 4, "v_weights": 5,
           "q0": 6, "qT": 7, "traj": 8, "pdf": 9, "times": 10, "D": 11, "proj": 12}


class Pipeline:
    """Oracle ComputePipeline (reference src/server/compute_pipeline.mojo)."""

    def __init__(self, kappa=1.2, theta=0.05, sigma=0.35, rho=-0.4, r=0.05, T=0.5, S0=100.0,
                 V0=0.1, n_s=38, n_v=38, barrier=0.0, option_type=9, s_min=0.0, s_max=-1.0,
                 opt: OrcOptions | None = None):
        self._L = lib()
        self._h = self._L.orc_create(kappa, theta, sigma, rho, r, T, S0, V0, n_s, n_v, barrier,
                                     option_type, s_min, s_max,
                                     C.byref(opt) if opt is not None else None)
        if not self._h:
            raise ValueError("invalid FPE parameters")

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.orc_destroy(self._h)
            self._h = None

    def array(self, what: str) -> np.ndarray:
        k = _ARRAYS[what]
        n = self._L.orc_len(self._h, k)
        out = np.empty(int(n), dtype=np.float64)
        self._L.orc_fill(self._h, k, _dp(out))
        return out

    def dims(self) -> dict:
        out = (C.c_int64 * 12)()
        self._L.orc_dims(self._h, out)
        keys = ["n_dof_s", "n_dof_v", "n_qs", "n_qv", "accepted", "rejected", "newton", "gmres",
                "lu", "admm", "success", "kl"]
        return dict(zip(keys, list(out)))

    def basis_csr(self, which: int):
        nr, nc = C.c_int32(), C.c_int32()
        nnz = self._L.orc_basis_csr(self._h, which, C.byref(nr), C.byref(nc), None, None, None)
        indptr = np.empty(nr.value + 1, np.int32)
        indices = np.empty(nnz, np.int32)
        data = np.empty(nnz, np.float64)
        ip = C.POINTER(C.c_int32)
        self._L.orc_basis_csr(self._h, which, C.byref(nr), C.byref(nc),
                              indptr.ctypes.data_as(ip), indices.ctypes.data_as(ip), _dp(data))
        return data, indices, indptr, (nr.value, nc.value)

    def factor(self, which: int) -> np.ndarray:
        n = self._L.orc_factor(self._h, which, None)
        out = np.empty((n, n), np.float64)
        self._L.orc_factor(self._h, which, _dp(out))
        return out

    def price_at(self, K) -> np.ndarray:
        K = np.ascontiguousarray(np.atleast_1d(np.asarray(K, np.float64)))
        out = np.empty_like(K)
        self._L.orc_price_at(self._h, _dp(K), len(K), _dp(out))
        return out

    def greeks(self, K, rel_s=0.0, rel_v=0.0):
        K = np.ascontiguousarray(np.atleast_1d(np.asarray(K, np.float64)))
        d, g, v = (np.empty_like(K) for _ in range(3))
        self._L.orc_greeks(self._h, _dp(K), len(K), rel_s, rel_v, _dp(d), _dp(g), _dp(v))
        return d, g, v


def pricer_price(kappa, theta, sigma, rho, r, T, S0, V0, K, barrier=0.0, option_type=8, n_s=38,
                 n_v=38, s_min=0.0, s_max=-1.0, opt: OrcOptions | None = None) -> np.ndarray:
    K = np.ascontiguousarray(np.atleast_1d(np.asarray(K, np.float64)))
    out = np.empty_like(K)
    lib().orc_pricer_price(kappa, theta, sigma, rho, r, T, S0, V0, n_s, n_v, barrier, option_type,
                           s_min, s_max, _dp(K), len(K),
                           C.byref(opt) if opt is not None else None, _dp(out))
    return out


def engine_price(kappa, theta, sigma, rho, r, T, S0, V0, K, barrier=0.0, option_type=8, n_s=38,
                 n_v=38, s_min=0.0, s_max=-1.0, opt: OrcOptions | None = None):
    K = np.ascontiguousarray(np.atleast_1d(np.asarray(K, np.float64)))
    p, d, g, v = (np.empty_like(K) for _ in range(4))
    rc = lib().orc_engine_price(kappa, theta, sigma, rho, r, T, S0, V0, n_s, n_v, barrier,
                                option_type, s_min, s_max, _dp(K), len(K),
                                C.byref(opt) if opt is not None else None,
                                _dp(p), _dp(d), _dp(g), _dp(v))
    return p, d, g, v, rc


def price_batch(params: np.ndarray, ints: np.ndarray, opt: OrcOptions | None = None,
                n_threads: int = 1) -> np.ndarray:
    params = np.ascontiguousarray(params, np.float64)
    ints = np.ascontiguousarray(ints, np.int32)
    out = np.empty(len(params), np.float64)
    lib().orc_price_batch(len(params), _dp(params), ints.ctypes.data_as(C.POINTER(C.c_int32)),
                          C.byref(opt) if opt is not None else None, n_threads, _dp(out))
    return out


def heston_cf(kappa, theta, sigma, rho, r, T, S0, V0, K, is_call=True) -> float:
    return lib().orc_heston_cf_price(kappa, theta, sigma, rho, r, T, S0, V0, K, int(is_call))


def bspline_value(knots, degree, x, i) -> float:
    k = np.ascontiguousarray(np.asarray(knots, np.float64))
    return lib().orc_bspline_value(_dp(k), len(k), degree, x, i)


def generate_knots(n, degree, nonuniform, center, b0, b1, mean, std) -> np.ndarray:
    out = np.empty(4 * n + 64, np.float64)
    m = lib().orc_generate_knots(n, degree, int(nonuniform), center, b0, b1, mean, std, _dp(out))
    return out[:m].copy()


def payoff(option_type, K, barrier, S) -> np.ndarray:
    K = np.ascontiguousarray(np.atleast_1d(np.asarray(K, np.float64)))
    out = np.empty_like(K)
    lib().orc_payoff(option_type, _dp(K), len(K), barrier, S, _dp(out))
    return out


def radau_dense(M, K, y0, t1, rtol, atol, max_step=0.0, first_step=0.0, exact=False):
    M = np.ascontiguousarray(M, np.float64)
    K = np.ascontiguousarray(K, np.float64)
    y0 = np.ascontiguousarray(y0, np.float64)
    out = np.empty_like(y0)
    n = lib().orc_radau_dense(len(y0), _dp(M), _dp(K), _dp(y0), t1, rtol, atol, max_step,
                              first_step, int(exact), _dp(out))
    return out, n


def pdf_interpolate(s_points, v_points, pdf, s, v) -> np.ndarray:
    sp = np.ascontiguousarray(s_points, np.float64)
    vp = np.ascontiguousarray(v_points, np.float64)
    f = np.ascontiguousarray(pdf, np.float64)
    sq = np.ascontiguousarray(np.atleast_1d(s), np.float64)
    vq = np.ascontiguousarray(np.atleast_1d(v), np.float64)
    out = np.empty(len(sq))
    rc = lib().orc_pdf_interpolate(_dp(sp), len(sp), _dp(vp), len(vp), _dp(f), _dp(sq), _dp(vq), len(sq), _dp(out))
    if rc != 0:
        raise ValueError("orc_pdf_interpolate: bad arguments")
    return out
