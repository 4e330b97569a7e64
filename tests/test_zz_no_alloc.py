"""The allocation-free entry point (fpe_price_noalloc) against the ordinary
batched entry point (fpe_price_batch), through the C ABI, on a GPU.

fpe_price_noalloc is for callers that cannot allocate device memory while
pricing (stream capture, fixed memory budgets, plug-ins in another
application's memory pool); it keeps all scratch in one static device array
that every call reuses.  Two calls in a row must give the same answers as
the allocating path, so leftovers from the previous call must not leak into
the next one.  This file is collected last; it also passes on its own.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

H = dict(kappa=1.2, theta=0.05, sigma=0.35, rho=-0.4, r=0.1, T=0.6, S0=60.0, V0=0.1)


def _contract(lib_mod, strikes, option_type, barrier, n_s, n_v, s_max=150.0):
    k = np.ascontiguousarray(strikes, dtype=np.float64)
    c = lib_mod.FpeContract(H["kappa"], H["theta"], H["sigma"], H["rho"], H["r"], H["T"],
                            H["S0"], H["V0"], barrier, 0.0, s_max, n_s, n_v, option_type, len(k),
                            k.ctypes.data_as(lib_mod.dp))
    return c, k


def _both(engine, strikes, option_type, barrier, n, opts):
    from fpe_option_b200 import _lib

    L = _lib.load()
    c, keep = _contract(_lib, strikes, option_type, barrier, n, n)
    o = opts.to_c()
    nk = len(strikes)
    ref = np.zeros(nk)
    ref_st = np.zeros(nk, np.int32)
    rc = L.fpe_price_batch(C.byref(c), 1, C.byref(o), ref.ctypes.data_as(_lib.dp), None, None,
                           None, ref_st.ctypes.data_as(_lib.ip))
    assert rc == 0 and (ref_st == 0).all()
    outs = []
    for _ in range(2):  # two calls in a row share the static scratch
        got = np.full(nk, np.nan)
        st = np.full(nk, -7, np.int32)
        rc = L.fpe_price_noalloc(C.byref(c), C.byref(o), got.ctypes.data_as(_lib.dp),
                                 st.ctypes.data_as(_lib.ip), None)
        assert rc == 0 and (st == 0).all()
        outs.append(got)
    del keep
    return ref, outs


@pytest.mark.parametrize("ot,barrier", [(8, 0.0), (2, 52.0), (0, 52.0)])
def test_noalloc_matches_batched_entry_point(engine, ot, barrier):
    fpe = engine
    opts = fpe.BatchOptions(num_insert=50)
    ref, outs = _both(fpe, [56.0, 60.0, 66.0], ot, barrier, 10, opts)
    for got in outs:
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-14)


def test_noalloc_mixed_precision_config(engine):
    fpe = engine
    opts = fpe.BatchOptions(disc=1, precision=1, rtol=1e-6, atol=1e-8)
    ref, outs = _both(fpe, [58.0, 61.0], 9, 0.0, 24, opts)
    for got in outs:
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-14)


def test_noalloc_rejects_oversized_grids(engine):
    from fpe_option_b200 import _lib

    L = _lib.load()
    c, keep = _contract(_lib, [60.0], 8, 0.0, 256, 60)
    o = engine.BatchOptions(num_insert=50).to_c()
    got = np.zeros(1)
    st = np.zeros(1, np.int32)
    rc = L.fpe_price_noalloc(C.byref(c), C.byref(o), got.ctypes.data_as(_lib.dp),
                             st.ctypes.data_as(_lib.ip), None)
    assert rc == -2 and st[0] == 1
    # the array is still usable afterwards
    ref, outs = _both(engine, [60.0], 8, 0.0, 8, engine.BatchOptions(num_insert=50))
    np.testing.assert_allclose(outs[1], ref, rtol=1e-12)
