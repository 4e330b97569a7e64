"""The allocation-free entry point (fpe_price_noalloc) against the ordinary
batched entry point (fpe_price_batch) and the CPU oracle, through the C ABI,
on a GPU.

fpe_price_noalloc is for callers that cannot allocate device memory while
pricing (hosts with a GPU memory budget fixed at start-up, plug-ins in
another application's memory pool); it keeps all scratch in one static
device array that every call reuses.  Two calls in a row must give the same
answers as the allocating path, so leftovers from the previous call must not
leak into the next one.  It copies its results to the host and waits, so on a
stream under graph capture it must refuse before enqueuing anything.  This
file is collected last; it also passes on its own.
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


def _both(engine, strikes, option_type, barrier, n, opts, n_v=None, s_max=150.0, stream=None):
    from fpe_option_b200 import _lib

    L = _lib.load()
    c, keep = _contract(_lib, strikes, option_type, barrier, n, n if n_v is None else n_v, s_max)
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
                                 st.ctypes.data_as(_lib.ip), stream)
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


def test_noalloc_default_domain_and_caller_stream(engine):
    """s_max = 0 (the 3 S0 default) on a stream the caller created."""
    import torch

    stream = torch.cuda.Stream()
    ref, outs = _both(engine, [57.0, 63.0], 9, 0.0, 10, engine.BatchOptions(num_insert=50), s_max=0.0,
                      stream=C.c_void_p(stream.cuda_stream))
    for got in outs:
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-14)


def test_noalloc_global_factor_scratch(engine):
    """48 v-dofs in mixed precision with full-width (48 x 48) stage-LU blocks:
    the factorization scratch does not fit in shared memory and lives in the
    static array (the kernel's global branch)."""
    opts = engine.BatchOptions(disc=1, precision=1, rtol=1e-6, atol=1e-8, block_split=1)
    ref, outs = _both(engine, [60.0], 8, 0.0, 16, opts, n_v=48)
    for got in outs:
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-14)


def test_noalloc_matches_the_oracle(engine, oracle):
    """The reference discretization in FP64 against the CPU oracle's Pricer."""
    from fpe_option_b200 import _lib

    L = _lib.load()
    strikes = [56.0, 62.0]
    c, keep = _contract(_lib, strikes, 0, 52.0, 10, 10)
    o = engine.BatchOptions(num_insert=50, complex_solve=1, radau_constants=1).to_c()
    got = np.zeros(2)
    st = np.zeros(2, np.int32)
    rc = L.fpe_price_noalloc(C.byref(c), C.byref(o), got.ctypes.data_as(_lib.dp), st.ctypes.data_as(_lib.ip), None)
    assert rc == 0 and (st == 0).all()
    exp = oracle.pricer_price(*H.values(), K=strikes, barrier=52.0, option_type=0, n_s=10, n_v=10, s_max=150.0,
                              opt=oracle.options(num_insert=50))
    np.testing.assert_allclose(got, exp, rtol=1e-9)


def test_noalloc_refuses_a_capturing_stream(engine):
    """A stream under graph capture gets FPE_NOALLOC_ERR_CAPTURE before anything
    is enqueued, and the capture stays valid."""
    import torch

    from fpe_option_b200 import _lib

    L = _lib.load()
    c, keep = _contract(_lib, [60.0], 8, 0.0, 10, 10)
    o = engine.BatchOptions(num_insert=50).to_c()
    got = np.zeros(1)
    st = np.zeros(1, np.int32)
    s = torch.cuda.Stream()
    sp = C.c_void_p(s.cuda_stream)
    assert L.fpe_price_noalloc(C.byref(c), C.byref(o), got.ctypes.data_as(_lib.dp),
                               st.ctypes.data_as(_lib.ip), sp) == 0  # device set-up outside capture
    x = torch.zeros(4, device="cuda")
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        rc = L.fpe_price_noalloc(C.byref(c), C.byref(o), got.ctypes.data_as(_lib.dp),
                                 st.ctypes.data_as(_lib.ip), sp)
        x += 1.0
    assert rc == -3
    g.replay()
    torch.cuda.synchronize()
    assert float(x[0]) == 1.0
    del g


def test_noalloc_second_device():
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("one CUDA device")
    from fpe_option_b200 import _lib

    L = _lib.load()
    c, keep = _contract(_lib, [60.0], 8, 0.0, 10, 10)
    o = _lib.FpeBatchOptions()
    o.num_insert = 50
    out = []
    for dev in (0, 1):
        torch.cuda.set_device(dev)
        got = np.zeros(1)
        st = np.zeros(1, np.int32)
        assert L.fpe_price_noalloc(C.byref(c), C.byref(o), got.ctypes.data_as(_lib.dp),
                                   st.ctypes.data_as(_lib.ip), None) == 0
        out.append(got[0])
    torch.cuda.set_device(0)
    assert out[0] == out[1]
