"""Surrogate pricer: a BF16 tensor-core MLP trained on prices from the batched
FPE solver (include/fpe_surrogate.h).

``Mlp`` wraps one network (forward, Adam training step, gradient).  The
surrogate in front of the pricer -- feature encoding, an ensemble, the input
box it was trained on, and the fall-back to the FPE solver -- is
``SurrogatePricer``.  Device memory comes from torch (plumbing only); all
arithmetic runs in the library's CUDA kernels.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("the surrogate needs a CUDA device")
    return torch


class Mlp:
    """n_in -> hidden x layers -> 1 SiLU network with BF16 tensor-core layers."""

    def __init__(self, n_in: int = 12, hidden: int = 256, layers: int = 4, max_rows: int = 4096,
                 seed: int = 0):
        self._L = _lib.load()
        self._h = self._L.fpe_mlp_create(n_in, hidden, layers, max_rows, seed)
        if not self._h:
            raise RuntimeError("fpe_mlp_create failed (bad shape or no CUDA device)")
        lay = (C.c_int32 * 4)()
        self.n_params = int(self._L.fpe_mlp_layout(self._h, lay))
        self.layout = tuple(int(v) for v in lay)
        self.max_rows = max_rows
        self._torch = _torch()

    # -- parameters ------------------------------------------------------------
    def get_params(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        if self._L.fpe_mlp_get_params(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), self.n_params):
            raise RuntimeError("fpe_mlp_get_params failed")
        return out

    def set_params(self, theta: np.ndarray) -> None:
        th = np.ascontiguousarray(theta, dtype=np.float32)
        if th.size != self.n_params or self._L.fpe_mlp_set_params(
                self._h, th.ctypes.data_as(C.POINTER(C.c_float)), self.n_params):
            raise RuntimeError("fpe_mlp_set_params failed")

    # -- device-tensor entry points --------------------------------------------
    def _stream(self, stream):
        """The CUDA stream for a call: the given one, else torch's current stream
        (its legacy default stream passed as cudaStreamLegacy), so that the
        library's kernels are ordered with the torch ops around them."""
        if stream is not None:
            return stream
        h = self._torch.cuda.current_stream().cuda_stream
        return h if h else 1  # cudaStreamLegacy

    def forward_dev(self, x, y, stream: int | None = None) -> None:
        """y[n] = net(x[n, n_in]) for float32 CUDA tensors."""
        n = int(x.shape[0])
        if self._L.fpe_mlp_forward(self._h, x.data_ptr(), n, y.data_ptr(), self._stream(stream)):
            raise RuntimeError("fpe_mlp_forward failed")

    def train_step_dev(self, x, t, w, lr: float, loss=None, stream: int | None = None) -> None:
        n = int(x.shape[0])
        rc = self._L.fpe_mlp_train_step(self._h, x.data_ptr(), t.data_ptr(),
                                        w.data_ptr() if w is not None else None, n, float(lr),
                                        loss.data_ptr() if loss is not None else None,
                                        self._stream(stream))
        if rc:
            raise RuntimeError("fpe_mlp_train_step failed")

    # -- host-array conveniences -------------------------------------------------
    def _dev(self, a):
        return self._torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device="cuda")

    def forward(self, x: np.ndarray) -> np.ndarray:
        tx = self._dev(x)
        ty = self._torch.empty(tx.shape[0], device="cuda")
        self.forward_dev(tx, ty)
        self._torch.cuda.synchronize()
        return ty.cpu().numpy().astype(np.float64)

    def train_step(self, x, t, w=None, lr: float = 1e-3) -> None:
        self.train_step_dev(self._dev(x), self._dev(t), None if w is None else self._dev(w), lr)
        self._torch.cuda.synchronize()

    def gradient(self, x, t, w=None):
        """(loss, gradient) of sum_i w_i (net(x_i) - t_i)^2 / n at the current parameters."""
        tx, tt = self._dev(x), self._dev(t)
        tw = None if w is None else self._dev(w)
        g = np.empty(self.n_params, np.float32)
        loss = C.c_float(0.0)
        self._torch.cuda.synchronize()  # the gradient call runs on the library's own stream
        rc = self._L.fpe_mlp_gradient(self._h, tx.data_ptr(), tt.data_ptr(),
                                      tw.data_ptr() if tw is not None else None, int(tx.shape[0]),
                                      g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss))
        if rc:
            raise RuntimeError(f"fpe_mlp_gradient failed ({rc})")
        return float(loss.value), g.astype(np.float64)

    def loss(self, x, t, w=None) -> float:
        e = self.forward(x) - np.asarray(t, np.float64)
        w = np.ones_like(e) if w is None else np.asarray(w, np.float64)
        return float(np.mean(w * e * e))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.fpe_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Surrogate pricer
# ---------------------------------------------------------------------------
# Box of the continuous inputs the surrogate is trained on: the parameter
# ranges of the batched workloads (kappa, theta, eta, rho, V0, r, T), strikes
# K/S0 in [0.7, 1.3] (calibration surfaces) and barriers B/S0 in [0, 1.4]
# (0 for Europeans; down barriers 0.6-0.95, up barriers 1.05-1.4).
FEATURE_NAMES = ("kappa", "theta", "eta", "rho", "V0", "r", "T", "K/S0", "B/S0",
                 "is_call", "is_knock_out", "is_knock_in")
BOX_LO = np.array([0.5, 0.02, 0.1, -0.9, 0.02, 0.0, 0.1, 0.7, 0.0])
BOX_HI = np.array([3.0, 0.15, 0.8, 0.0, 0.2, 0.05, 2.0, 1.3, 1.4])
# option types the surrogate covers: European call/put, down-and-out/in calls,
# up-and-out/in puts
SURROGATE_TYPES = (8, 9, 2, 0, 7, 5)
# The network predicts y = log(price / S0 + LOG_EPS): squared error in y is a
# relative-price error floored at LOG_EPS S0, and the BF16 rounding of the
# activations (about 2^-9 relative) becomes a uniform relative price error
# instead of an absolute one that would swamp small prices.
LOG_EPS = 1e-3


def encode(params: np.ndarray, ints: np.ndarray):
    """(features (n, 12) float32 in [-1, 1] inside the box, in_box mask).

    params / ints use the package's contract tables (contracts_from_arrays):
    [kappa theta sigma rho r T S0 V0 K barrier s_min s_max] and [n_s n_v type].
    """
    P = np.asarray(params, np.float64)
    t = np.asarray(ints)[:, 2].astype(int)
    S0 = P[:, 6]
    cont = np.stack([P[:, 0], P[:, 1], P[:, 2], P[:, 3], P[:, 7], P[:, 4], P[:, 5],
                     P[:, 8] / S0, P[:, 9] / S0], axis=1)
    x = 2.0 * (cont - BOX_LO) / (BOX_HI - BOX_LO) - 1.0
    is_call = (t % 2 == 0).astype(np.float64)
    is_out = np.isin(t, (2, 3, 6, 7)).astype(np.float64)
    is_in = np.isin(t, (0, 1, 4, 5)).astype(np.float64)
    feats = np.concatenate([x, is_call[:, None], is_out[:, None], is_in[:, None]], axis=1)
    in_box = np.all(np.abs(x) <= 1.0 + 1e-9, axis=1) & np.isin(t, SURROGATE_TYPES)
    return feats.astype(np.float32), in_box


def draw_contracts(n: int, seed: int, kind: str = "european", grid=(48, 24)):
    """Seeded contracts over the surrogate's box, in the package's tables.

    kind "european": calls/puts 50/50, K/S0 ~ U[0.7, 1.3]; "barrier": down-
    and-out/in calls with B/S0 ~ U[0.6, 0.95] and up-and-out/in puts with
    B/S0 ~ U[1.05, 1.4], K/S0 ~ U[0.8, 1.2]; "mixed": half of each.  Heston
    parameters as the batched workloads draw them; S0 = 100, s_max = 3 S0.
    """
    rng = np.random.default_rng(seed)
    P = np.zeros((n, 12))
    I = np.zeros((n, 3), np.int32)
    P[:, 0] = rng.uniform(0.5, 3.0, n)
    P[:, 1] = rng.uniform(0.02, 0.15, n)
    P[:, 2] = rng.uniform(0.1, 0.8, n)
    P[:, 3] = rng.uniform(-0.9, 0.0, n)
    P[:, 4] = rng.uniform(0.0, 0.05, n)
    P[:, 5] = rng.uniform(0.1, 2.0, n)
    P[:, 6] = 100.0
    P[:, 7] = rng.uniform(0.02, 0.2, n)
    P[:, 11] = 300.0
    I[:, 0], I[:, 1] = grid
    if kind == "mixed":
        half = n // 2
        a, ia = draw_contracts(half, seed, "european", grid)
        b, ib = draw_contracts(n - half, seed + 1, "barrier", grid)
        return np.concatenate([a, b]), np.concatenate([ia, ib])
    if kind == "european":
        P[:, 8] = 100.0 * rng.uniform(0.7, 1.3, n)
        I[:, 2] = np.where(rng.random(n) < 0.5, 8, 9)
    elif kind == "barrier":
        P[:, 8] = 100.0 * rng.uniform(0.8, 1.2, n)
        down = rng.random(n) < 0.5
        knock_in = rng.random(n) < 0.5
        P[:, 9] = np.where(down, 100.0 * rng.uniform(0.6, 0.95, n), 100.0 * rng.uniform(1.05, 1.4, n))
        I[:, 2] = np.where(down, np.where(knock_in, 0, 2), np.where(knock_in, 5, 7))
    else:
        raise ValueError(f"unknown kind {kind!r}")
    return P, I


@dataclass
class SurrogateConfig:
    members: int = 3
    hidden: int = 256
    layers: int = 4
    batch: int = 4096
    lr: float = 1e-3       # peak learning rate, cosine-decayed to zero over the run
    epochs: int = 200
    disagreement_tol: float = 1e-3  # relative spread of the members that sends a query to the FPE solver
    seed: int = 0


class SurrogatePricer:
    """An ensemble of BF16 tensor-core MLPs in front of the FPE solver.

    ``price(params, ints)`` answers from the ensemble mean where the query lies
    in the training box and the members agree to ``disagreement_tol``; every
    other query is priced by the batched FPE solver with ``fpe_options``.
    """

    def __init__(self, config: SurrogateConfig | None = None, fpe_options=None):
        from . import BatchOptions

        self.config = config or SurrogateConfig()
        self.fpe_options = fpe_options or BatchOptions(disc=1, precision=1, rtol=1e-6, atol=1e-8,
                                                       complex_solve=2, radau_constants=2)
        c = self.config
        self.members = [Mlp(12, c.hidden, c.layers, max(c.batch, 128), seed=c.seed + 101 * k)
                        for k in range(c.members)]
        self._torch = _torch()

    # -- data ---------------------------------------------------------------------
    def fpe_prices(self, params, ints) -> np.ndarray:
        """Prices from the batched FPE solver (raises if any solve failed)."""
        from . import price_batch

        p, st = price_batch(params, ints, self.fpe_options)
        if np.any(st != 0):
            raise RuntimeError(f"FPE solves failed with status {sorted(set(st[st != 0].tolist()))}")
        return p

    @staticmethod
    def targets(params, prices):
        """Training targets log(price / S0 + LOG_EPS) and unit weights."""
        y = np.asarray(prices, np.float64) / np.asarray(params, np.float64)[:, 6]
        y = np.log(np.maximum(y, 0.0) + LOG_EPS)
        return y, np.ones_like(y)

    @staticmethod
    def to_price(y, S0):
        return np.asarray(S0) * (np.exp(np.asarray(y, np.float64)) - LOG_EPS)

    # -- training -------------------------------------------------------------------
    def fit(self, params, ints, prices, epochs: int | None = None, log=None) -> list[float]:
        """Adam on the relative squared error; returns the last epoch loss per member."""
        torch = self._torch
        c = self.config
        epochs = c.epochs if epochs is None else epochs
        x, _ = encode(params, ints)
        y, w = self.targets(params, prices)
        tx = torch.as_tensor(x, device="cuda")
        ty = torch.as_tensor(y.astype(np.float32), device="cuda")
        tw = torch.as_tensor(w.astype(np.float32), device="cuda")
        n = len(x)
        bs = min(c.batch, n)
        steps = max(1, epochs * (n // bs))
        losses = []
        for k, net in enumerate(self.members):
            gen = torch.Generator(device="cuda")
            gen.manual_seed(c.seed * 7919 + k)
            loss = torch.zeros(1, device="cuda")
            step = 0
            for ep in range(epochs):
                perm = torch.randperm(n, device="cuda", generator=gen)
                acc = torch.zeros(1, device="cuda")
                nb = 0
                for s in range(0, n - bs + 1, bs):
                    idx = perm[s:s + bs]
                    lr = 0.5 * c.lr * (1.0 + np.cos(np.pi * step / steps))
                    step += 1
                    net.train_step_dev(tx[idx].contiguous(), ty[idx].contiguous(), tw[idx].contiguous(),
                                       lr, loss)
                    acc += loss
                    nb += 1
                if log is not None and (ep + 1) % max(1, epochs // 5) == 0:
                    log(f"member {k} epoch {ep + 1}: loss {float(acc.item()) / max(nb, 1):.3e}")
            losses.append(float(acc.item()) / max(nb, 1))
        torch.cuda.synchronize()
        return losses

    # -- inference --------------------------------------------------------------------
    def predict_features(self, x_dev):
        """(mean log-price target, spread) of the members for a float32 CUDA
        feature tensor; the spread max - min of the log targets is the members'
        relative price disagreement."""
        torch = self._torch
        n = int(x_dev.shape[0])
        outs = torch.empty((len(self.members), n), device="cuda")
        for k, net in enumerate(self.members):
            net.forward_dev(x_dev, outs[k])
        mean = outs.mean(0)
        spread = outs.max(0).values - outs.min(0).values
        return mean, spread

    def price(self, params, ints):
        """(prices, from_fpe mask): the surrogate where it is trusted, FPE elsewhere."""
        torch = self._torch
        P = np.asarray(params, np.float64)
        x, in_box = encode(P, ints)
        mean, spread = self.predict_features(torch.as_tensor(x, device="cuda"))
        y = mean.cpu().numpy().astype(np.float64)
        ok = in_box & (spread.cpu().numpy() <= self.config.disagreement_tol)
        prices = self.to_price(y, P[:, 6])
        fb = ~ok
        if np.any(fb):
            prices[fb] = self.fpe_prices(P[fb], np.asarray(ints)[fb])
        return prices, fb

    def close(self):
        for m in self.members:
            m.close()
