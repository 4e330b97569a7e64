"""CPU oracle of the surrogate MLP (test infrastructure only).

Restates, in float64 numpy, the network of include/fpe_surrogate.h: hidden
layers z = x W^T + b, h = SiLU(z), output y = h . w_out + b_out, loss
sum_i w_i (y_i - t_i)^2 / n, and its gradient -- with the BF16 roundings the
device applies at the same points (weights, inputs and activations entering
a tensor-core product, and the layer gradients that enter the next product),
so that the device forward/backward can be checked value by value.  The Adam
step follows the reference update rule (src/nn/adam.mojo:31-64).  Only
tests/ use this module; the product never does.
"""
from __future__ import annotations

import numpy as np


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    nan = np.isnan(f)
    out[nan] = np.nan
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def unpack(theta: np.ndarray, layout):
    """(Ws, bs, w_out, b_out) from the flat FP32 parameter vector."""
    n_in, in_pad, hidden, layers = layout
    o = 0
    Ws, bs = [], []
    for l in range(layers):
        fin = in_pad if l == 0 else hidden
        Ws.append(theta[o:o + hidden * fin].reshape(hidden, fin).astype(np.float64))
        o += hidden * fin
        bs.append(theta[o:o + hidden].astype(np.float64))
        o += hidden
    w_out = theta[o:o + hidden].astype(np.float64)
    o += hidden
    b_out = float(theta[o])
    return Ws, bs, w_out, b_out


def _ident(x):
    return np.asarray(x, dtype=np.float64)


def forward(theta, layout, x, keep=False, exact=False):
    """Network output; exact=True drops the BF16 roundings (plain float64)."""
    rnd = _ident if exact else bf16
    n_in, in_pad, hidden, layers = layout
    Ws, bs, w_out, b_out = unpack(theta, layout)
    X = np.zeros((x.shape[0], in_pad))
    X[:, :n_in] = x
    h = rnd(X)
    zs, hs = [], [h]
    for l in range(layers):
        z = h @ rnd(Ws[l]).T + bs[l]
        if not exact:
            z = z.astype(np.float32).astype(np.float64)
        h = rnd(silu(z))
        zs.append(z)
        hs.append(h)
    y = h @ w_out + b_out
    return (y, zs, hs) if keep else y


def gradient(theta, layout, x, t, w=None, exact=False):
    """(loss, flat gradient) of sum_i w_i (y_i - t_i)^2 / n."""
    rnd = _ident if exact else bf16
    n_in, in_pad, hidden, layers = layout
    Ws, bs, w_out, b_out = unpack(theta, layout)
    y, zs, hs = forward(theta, layout, x, keep=True, exact=exact)
    n = x.shape[0]
    w = np.ones(n) if w is None else np.asarray(w, dtype=np.float64)
    e = y - t
    loss = float(np.sum(w * e * e) / n)
    dy = 2.0 * w * e / n
    g_wout = hs[-1].T @ dy
    g_bout = dy.sum()
    dZ = np.outer(dy, w_out) * dsilu(zs[-1])
    gW = [None] * layers
    gb = [None] * layers
    for l in range(layers - 1, -1, -1):
        dZb = rnd(dZ)
        gW[l] = dZb.T @ hs[l]
        gb[l] = dZ.sum(axis=0)
        if l > 0:
            dH = dZb @ rnd(Ws[l])
            dZ = dH * dsilu(zs[l - 1])
    parts = []
    for l in range(layers):
        parts += [gW[l].ravel(), gb[l]]
    parts += [g_wout, np.array([g_bout])]
    return loss, np.concatenate(parts)


def adam_step(theta, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return theta - lr * mh / (np.sqrt(vh) + eps), m, v
