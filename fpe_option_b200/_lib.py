"""ctypes binding of ``libfpe_engine.so`` (the C ABI in include/fpe_engine.h and
include/fpe_surrogate.h).

The library is built in-tree by :func:`fpe_option_b200.build.build_library`.
There is no CPU fallback: loading fails loudly when the shared object is
missing, and every compute entry point reports failure without a GPU.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfpe_engine.so")

d, i32, i64, vp = C.c_double, C.c_int32, C.c_int64, C.c_void_p
dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int32)


class FpeVecResult(C.Structure):
    _fields_ = [("data", dp), ("len", i32)]


class FpeVec2Result(C.Structure):
    _fields_ = [("s_data", dp), ("s_len", i32), ("v_data", dp), ("v_len", i32)]


class FpeGridPtsResult(C.Structure):
    _fields_ = [("s_data", dp), ("s_len", i32), ("v_data", dp), ("v_len", i32),
                ("sw_data", dp), ("vw_data", dp)]


class FpeMatResult(C.Structure):
    _fields_ = [("data", dp), ("n_rows", i32), ("n_cols", i32)]


class FpeGreeksResult(C.Structure):
    _fields_ = [("delta", dp), ("gamma", dp), ("vega", dp), ("len", i32)]


class FpeOneshotResult(C.Structure):
    _fields_ = [("price", dp), ("delta", dp), ("gamma", dp), ("vega", dp), ("len", i32)]


class FpeContract(C.Structure):
    _fields_ = [("kappa", d), ("theta", d), ("sigma", d), ("rho", d), ("r", d), ("T", d),
                ("S0", d), ("V0", d), ("barrier", d), ("s_min", d), ("s_max", d),
                ("n_s", i32), ("n_v", i32), ("option_type", i32), ("n_strikes", i32),
                ("strikes", dp)]


class FpeBatchOptions(C.Structure):
    _fields_ = [("disc", i32), ("precision", i32), ("num_insert", i32), ("refine", i32),
                ("rtol", d), ("atol", d), ("ic_sigma_s", d), ("ic_sigma_v", d), ("ic_sub", i32),
                ("greeks", i32), ("rel_s", d), ("rel_v", d), ("complex_solve", i32),
                ("radau_constants", i32), ("max_step", d), ("first_step", d),
                ("price_rule", i32), ("max_steps", i32), ("fp64_retry", i32),
                ("stage_wait_cycles", i64), ("block_split", i32), ("sweep_buffers", i32),
                ("knock_in_tol_scale", d)]


# Every symbol declared in include/*.h.
EXPORTED = [
    "fpe_compute_create", "fpe_compute_destroy", "fpe_compute_knots", "fpe_compute_grid_points",
    "fpe_compute_initial_condition", "fpe_compute_solve", "fpe_compute_pdf", "fpe_compute_price",
    "fpe_compute_greeks", "fpe_price_oneshot", "fpe_compute_free_vec", "fpe_compute_free_vec2",
    "fpe_compute_free_grid_pts", "fpe_compute_free_mat", "fpe_compute_free_greeks",
    "fpe_compute_free_oneshot", "fpe_plan_create", "fpe_plan_run", "fpe_plan_results",
    "fpe_plan_stats", "fpe_plan_sizes", "fpe_plan_destroy", "fpe_price_batch",
    "fpe_compute_create_ex", "fpe_compute_basis_csr", "fpe_device_available",
    "fpe_plan_kernel_times", "fpe_plan_retried", "fpe_plan_solve_info", "fpe_tune_set", "fpe_tune_get",
    "fpe_tune_clear", "fpe_price_noalloc", "fpe_heston_cf_batch", "fpe_heston_cf_price",
    "fpe_pdf_interpolate",
    # include/fpe_surrogate.h
    "fpe_mlp_create", "fpe_mlp_destroy", "fpe_mlp_layout", "fpe_mlp_get_params",
    "fpe_mlp_set_params", "fpe_mlp_forward", "fpe_mlp_train_step", "fpe_mlp_gradient",
    "fpe_mlp_set_lr_schedule",
    "fpe_gemm_bf16",
]

_lib = None


def load():
    """Load the library (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"libfpe_engine.so not built ({LIB_PATH}); run fpe_option_b200.build.build_library()")
    L = C.CDLL(LIB_PATH)
    cp = vp
    L.fpe_compute_create.restype = cp
    L.fpe_compute_create.argtypes = [d] * 8 + [i32, i32, d, i32, i32, d, d]
    L.fpe_compute_create_ex.restype = cp
    L.fpe_compute_create_ex.argtypes = [d] * 8 + [i32, i32, d, i32, d, d,
                                                  C.POINTER(FpeBatchOptions)]
    L.fpe_compute_destroy.argtypes = [cp]
    L.fpe_compute_knots.argtypes = [cp, C.POINTER(FpeVec2Result)]
    L.fpe_compute_grid_points.argtypes = [cp, C.POINTER(FpeGridPtsResult)]
    L.fpe_compute_initial_condition.argtypes = [cp, C.POINTER(FpeVecResult)]
    L.fpe_compute_solve.argtypes = [cp, C.POINTER(FpeMatResult)]
    L.fpe_compute_pdf.argtypes = [cp, C.POINTER(FpeMatResult)]
    L.fpe_compute_price.argtypes = [cp, dp, i32, C.POINTER(FpeVecResult)]
    L.fpe_compute_greeks.argtypes = [cp, dp, i32, d, d, C.POINTER(FpeGreeksResult)]
    L.fpe_price_oneshot.argtypes = [d] * 8 + [dp, i32, d, i32, i32, i32, i32, d, d,
                                              C.POINTER(FpeOneshotResult)]
    L.fpe_compute_free_vec.argtypes = [C.POINTER(FpeVecResult)]
    L.fpe_compute_free_vec2.argtypes = [C.POINTER(FpeVec2Result)]
    L.fpe_compute_free_grid_pts.argtypes = [C.POINTER(FpeGridPtsResult)]
    L.fpe_compute_free_mat.argtypes = [C.POINTER(FpeMatResult)]
    L.fpe_compute_free_greeks.argtypes = [C.POINTER(FpeGreeksResult)]
    L.fpe_compute_free_oneshot.argtypes = [C.POINTER(FpeOneshotResult)]
    L.fpe_plan_create.restype = cp
    L.fpe_plan_create.argtypes = [C.POINTER(FpeContract), i32, C.POINTER(FpeBatchOptions)]
    L.fpe_plan_run.restype = i32
    L.fpe_plan_run.argtypes = [cp, vp]
    L.fpe_plan_results.restype = i32
    L.fpe_plan_results.argtypes = [cp, dp, dp, dp, dp, ip]
    L.fpe_plan_stats.restype = i32
    L.fpe_plan_stats.argtypes = [cp, C.POINTER(C.c_int64)]
    L.fpe_plan_kernel_times.restype = i32
    L.fpe_plan_kernel_times.argtypes = [cp, vp, C.POINTER(C.c_float)]
    L.fpe_plan_sizes.restype = i32
    L.fpe_plan_sizes.argtypes = [cp, ip, ip]
    L.fpe_plan_retried.restype = i32
    L.fpe_plan_retried.argtypes = [cp]
    L.fpe_plan_solve_info.restype = i32
    L.fpe_plan_solve_info.argtypes = [cp, ip]
    L.fpe_tune_set.restype = i32
    L.fpe_tune_set.argtypes = [i32] * 7
    L.fpe_tune_get.restype = i32
    L.fpe_tune_get.argtypes = [i32] * 5 + [ip, ip]
    L.fpe_tune_clear.restype = None
    L.fpe_tune_clear.argtypes = []
    L.fpe_plan_destroy.argtypes = [cp]
    L.fpe_price_batch.restype = i32
    L.fpe_price_batch.argtypes = [C.POINTER(FpeContract), i32, C.POINTER(FpeBatchOptions),
                                  dp, dp, dp, dp, ip]
    L.fpe_compute_basis_csr.restype = i64
    L.fpe_compute_basis_csr.argtypes = [cp, i32, ip, ip, ip, ip, dp]
    L.fpe_device_available.restype = i32
    L.fpe_device_available.argtypes = []
    fp = C.POINTER(C.c_float)
    L.fpe_mlp_create.restype = vp
    L.fpe_mlp_create.argtypes = [i32, i32, i32, i32, C.c_uint64]
    L.fpe_mlp_destroy.argtypes = [vp]
    L.fpe_mlp_layout.restype = i64
    L.fpe_mlp_layout.argtypes = [vp, ip]
    L.fpe_mlp_get_params.restype = i32
    L.fpe_mlp_get_params.argtypes = [vp, fp, i64]
    L.fpe_mlp_set_params.restype = i32
    L.fpe_mlp_set_params.argtypes = [vp, fp, i64]
    L.fpe_mlp_forward.restype = i32
    L.fpe_mlp_forward.argtypes = [vp, vp, i32, vp, vp]
    L.fpe_mlp_train_step.restype = i32
    L.fpe_mlp_train_step.argtypes = [vp, vp, vp, vp, i32, C.c_float, vp, vp]
    L.fpe_mlp_gradient.restype = i32
    L.fpe_mlp_gradient.argtypes = [vp, vp, vp, vp, i32, fp, fp]
    L.fpe_mlp_set_lr_schedule.restype = i32
    L.fpe_mlp_set_lr_schedule.argtypes = [vp, fp, i32]
    L.fpe_gemm_bf16.restype = i32
    L.fpe_gemm_bf16.argtypes = [vp, i32, vp, i32, i32, i32, i32, vp, i32, vp, i32, vp]
    L.fpe_price_noalloc.restype = i32
    L.fpe_price_noalloc.argtypes = [C.POINTER(FpeContract), C.POINTER(FpeBatchOptions), dp, ip, vp]
    L.fpe_heston_cf_batch.restype = i32
    L.fpe_heston_cf_batch.argtypes = [vp, vp, vp, i32, vp, vp]
    L.fpe_heston_cf_price.restype = i32
    L.fpe_heston_cf_price.argtypes = [C.POINTER(FpeContract), i32, dp, ip]
    L.fpe_pdf_interpolate.restype = i32
    L.fpe_pdf_interpolate.argtypes = [vp, i32, vp, i32, vp, vp, vp, i32, vp, vp]
    _lib = L
    return L
