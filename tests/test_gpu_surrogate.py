"""Surrogate MLP on the GPU: the tensor-core BF16 product against float64
numpy on the same BF16-rounded inputs, the network's forward and gradient
against the CPU oracle (oracle/mlp_oracle.py, same roundings), and training.

Tolerances: products accumulate in FP32 over K <= 256 terms, so they match to
1e-4 of the operand scale.  The network's BF16 activations can round to the
neighbouring BF16 value where the FP32 device sum and the float64 oracle sum
straddle a rounding boundary, so outputs match to 1e-2 relative and gradient
blocks to 3e-2 in norm.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    assert torch.cuda.is_available()
    return torch


def _bf16_tensor(torch, a):
    return torch.tensor(a, dtype=torch.float32, device="cuda").to(torch.bfloat16).contiguous()


# K a multiple of 64 takes the persistent TMA product (51200 rows: 400 tiles,
# so CTAs loop over several tiles and both TMEM accumulators), K = 16 the
# per-tile product.
@pytest.mark.parametrize("M,N,K,bias,act", [(256, 256, 256, False, 0), (128, 16, 256, False, 0),
                                            (384, 48, 16, True, 1), (128, 512, 64, True, 0),
                                            (256, 256, 4096, False, 0), (51200, 256, 256, True, 1),
                                            (640, 144, 128, True, 0)])
def test_tensor_core_gemm_matches_cpu(engine, M, N, K, bias, act):
    from fpe_option_b200 import _lib
    from oracle.mlp_oracle import bf16, silu

    torch = _torch()
    L = _lib.load()
    rng = np.random.default_rng(M + N + K)
    A = rng.standard_normal((M, K)).astype(np.float32)
    B = rng.standard_normal((N, K)).astype(np.float32)
    b = rng.standard_normal(N).astype(np.float32) if bias else None
    tA, tB = _bf16_tensor(torch, A), _bf16_tensor(torch, B)
    tb = torch.tensor(b, device="cuda") if bias else None
    out = torch.full((M, N), float("nan"), device="cuda")
    rc = L.fpe_gemm_bf16(tA.data_ptr(), K, tB.data_ptr(), K, M, N, K,
                         tb.data_ptr() if bias else None, act, out.data_ptr(), N, None)
    assert rc == 0
    ref = bf16(A) @ bf16(B).T
    if bias:
        ref = ref + b
    if act:
        ref = silu(ref)
    got = out.cpu().numpy()
    scale = np.sqrt(K)
    np.testing.assert_allclose(got, ref, rtol=1e-4, atol=1e-4 * scale)


def test_gemm_rejects_bad_shapes(engine):
    from fpe_option_b200 import _lib

    torch = _torch()
    L = _lib.load()
    a = torch.zeros((128, 32), dtype=torch.bfloat16, device="cuda")
    c = torch.zeros((128, 32), device="cuda")
    assert L.fpe_gemm_bf16(a.data_ptr(), 32, a.data_ptr(), 32, 100, 32, 32, None, 0, c.data_ptr(), 32, None) < 0
    assert L.fpe_gemm_bf16(a.data_ptr(), 32, a.data_ptr(), 32, 128, 24, 32, None, 0, c.data_ptr(), 32, None) < 0


def _mlp(n_in=12, hidden=256, layers=4, rows=512, seed=7):
    from fpe_option_b200.surrogate import Mlp

    return Mlp(n_in=n_in, hidden=hidden, layers=layers, max_rows=rows, seed=seed)


def test_mlp_forward_matches_oracle(engine):
    from oracle import mlp_oracle as mo

    rng = np.random.default_rng(11)
    net = _mlp()
    theta = net.get_params()
    x = rng.uniform(-1, 1, (300, 12)).astype(np.float32)
    got = net.forward(x)
    ref = mo.forward(theta, net.layout, x)
    assert np.max(np.abs(got - ref)) <= 1e-2 * max(1.0, np.max(np.abs(ref)))
    # inference splits inputs larger than max_rows
    x2 = rng.uniform(-1, 1, (1300, 12)).astype(np.float32)
    np.testing.assert_allclose(net.forward(x2), mo.forward(theta, net.layout, x2), atol=1e-2)


def test_mlp_gradient_matches_oracle(engine):
    from oracle import mlp_oracle as mo

    rng = np.random.default_rng(5)
    net = _mlp(rows=256)
    theta = net.get_params()
    x = rng.uniform(-1, 1, (256, 12)).astype(np.float32)
    t = rng.uniform(0, 0.3, 256).astype(np.float32)
    w = rng.uniform(0.5, 2.0, 256).astype(np.float32)
    loss, g = net.gradient(x, t, w)
    loss_ref, g_ref = mo.gradient(theta, net.layout, x, t, w)
    assert abs(loss - loss_ref) <= 1e-2 * loss_ref
    n_in, in_pad, hidden, layers = net.layout
    o = 0
    blocks = []
    for l in range(layers):
        fin = in_pad if l == 0 else hidden
        blocks += [(f"W{l}", hidden * fin), (f"b{l}", hidden)]
    blocks += [("w_out", hidden), ("b_out", 1)]
    for name, size in blocks:
        a, b = g[o:o + size], g_ref[o:o + size]
        o += size
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert err < 3e-2, (name, err)
    # padded input columns get no gradient
    W0 = g[: hidden * in_pad].reshape(hidden, in_pad)
    assert np.all(W0[:, n_in:] == 0.0)


def test_adam_step_matches_oracle(engine):
    from oracle import mlp_oracle as mo

    rng = np.random.default_rng(9)
    net = _mlp(rows=128)
    theta = net.get_params().astype(np.float64)
    x = rng.uniform(-1, 1, (128, 12)).astype(np.float32)
    t = rng.uniform(0, 0.3, 128).astype(np.float32)
    _, g = net.gradient(x, t)
    net.train_step(x, t, lr=1e-3)
    th_ref, _, _ = mo.adam_step(theta, g.astype(np.float64), np.zeros_like(theta), np.zeros_like(theta), 1, 1e-3)
    np.testing.assert_allclose(net.get_params(), th_ref, rtol=0, atol=2e-6)


def test_training_fits_a_smooth_function(engine):
    rng = np.random.default_rng(2)
    net = _mlp(rows=1024, seed=3)
    x = rng.uniform(-1, 1, (1024, 12)).astype(np.float32)
    t = (0.2 + 0.1 * np.sin(2 * x[:, 0]) * x[:, 1] + 0.05 * x[:, 2] ** 2).astype(np.float32)
    first = net.loss(x, t)
    for _ in range(300):
        net.train_step(x, t, lr=1e-3)
    last = net.loss(x, t)
    assert last < 0.05 * first, (first, last)
