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

    def set_lr_schedule(self, table) -> None:
        """Per-step learning rates used by train steps given lr < 0."""
        t = np.ascontiguousarray(table, dtype=np.float32)
        if self._L.fpe_mlp_set_lr_schedule(self._h, t.ctypes.data_as(C.POINTER(C.c_float)), int(t.size)):
            raise RuntimeError("fpe_mlp_set_lr_schedule failed")

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
# The network predicts y = log(v / S0 + LOG_EPS), v the option's value above
# its discounted intrinsic value for Europeans (price - (S0 - K e^{-rT})+ for
# calls, price - (K e^{-rT} - S0)+ for puts) and the price itself for barrier
# options: squared error in y is a relative error of the part of the price
# that depends on the model, floored at LOG_EPS S0, and the BF16 rounding of
# the activations (about 2^-9 relative) becomes a relative error of that part
# instead of an absolute one that would swamp small or deep in-the-money prices.
LOG_EPS = 1e-3


def intrinsic(params, ints) -> np.ndarray:
    """Discounted intrinsic value of European quotes (zero for other types)."""
    P = np.asarray(params, np.float64)
    t = np.asarray(ints)[:, 2]
    fwd = P[:, 8] * np.exp(-P[:, 4] * P[:, 5])
    call = np.maximum(P[:, 6] - fwd, 0.0)
    put = np.maximum(fwd - P[:, 6], 0.0)
    return np.where(t == 8, call, np.where(t == 9, put, 0.0))


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
        # the networks learn standardised targets (y - mu) / sd, fixed at fit()
        self.mu, self.sd = 0.0, 1.0

    # -- data ---------------------------------------------------------------------
    def fpe_prices(self, params, ints) -> np.ndarray:
        """Prices from the batched FPE solver (raises if any solve failed)."""
        from . import price_batch

        p, st = price_batch(params, ints, self.fpe_options)
        if np.any(st != 0):
            raise RuntimeError(f"FPE solves failed with status {sorted(set(st[st != 0].tolist()))}")
        return p

    @staticmethod
    def targets(params, ints, prices):
        """Training targets log(v / S0 + LOG_EPS) (v: see LOG_EPS) and unit weights."""
        P = np.asarray(params, np.float64)
        v = (np.asarray(prices, np.float64) - intrinsic(P, ints)) / P[:, 6]
        y = np.log(np.maximum(v, 0.0) + LOG_EPS)
        return y, np.ones_like(y)

    @staticmethod
    def to_price(y, params, ints):
        P = np.asarray(params, np.float64)
        return P[:, 6] * (np.exp(np.asarray(y, np.float64)) - LOG_EPS) + intrinsic(P, ints)

    # -- training -------------------------------------------------------------------
    def fit(self, params, ints, prices, epochs: int | None = None, log=None) -> list[float]:
        """Adam on the squared error of the standardised log-price targets;
        returns the last epoch's mean loss per member.

        One epoch -- the batch gathers and the training steps of every batch --
        is captured once as a CUDA graph per member and replayed each epoch with
        a fresh permutation; the cosine learning-rate schedule is read on the
        device by the step counter, so every replay trains with the right rate."""
        torch = self._torch
        c = self.config
        epochs = c.epochs if epochs is None else epochs
        x, _ = encode(params, ints)
        y, w = self.targets(params, ints, prices)
        self.mu, self.sd = float(y.mean()), float(max(y.std(), 1e-12))
        y = (y - self.mu) / self.sd
        tx = torch.as_tensor(x, device="cuda")
        ty = torch.as_tensor(y.astype(np.float32), device="cuda")
        tw = torch.as_tensor(w.astype(np.float32), device="cuda")
        n = len(x)
        bs = min(c.batch, n)
        nb = n // bs
        steps = max(1, epochs * nb)
        sched = 0.5 * c.lr * (1.0 + np.cos(np.pi * np.arange(steps) / steps))
        losses = []
        for k, net in enumerate(self.members):
            net.set_lr_schedule(sched)
            gen = torch.Generator(device="cuda")
            gen.manual_seed(c.seed * 7919 + k)
            perm = torch.zeros(nb * bs, dtype=torch.long, device="cuda")
            loss = torch.zeros(1, device="cuda")
            acc = torch.zeros(1, device="cuda")
            torch.cuda.synchronize()
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                acc.zero_()
                for b in range(nb):
                    idx = perm[b * bs:(b + 1) * bs]
                    net.train_step_dev(tx.index_select(0, idx), ty.index_select(0, idx),
                                       tw.index_select(0, idx), -1.0, loss)
                    acc += loss
            for ep in range(epochs):
                perm.copy_(torch.randperm(n, device="cuda", generator=gen)[:nb * bs])
                graph.replay()
                if log is not None and (ep + 1) % max(1, epochs // 5) == 0:
                    log(f"member {k} epoch {ep + 1}: loss {float(acc.item()) / nb:.3e}")
            torch.cuda.synchronize()
            losses.append(float(acc.item()) / nb)
            del graph
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
        mean = outs.mean(0) * self.sd + self.mu
        spread = (outs.max(0).values - outs.min(0).values) * self.sd
        return mean, spread

    def price(self, params, ints, gate_disagreement: bool = True):
        """(prices, from_fpe mask): the surrogate where it is trusted, FPE elsewhere.
        Trusted = inside the training box and, with gate_disagreement, members
        agreeing to disagreement_tol."""
        torch = self._torch
        P = np.asarray(params, np.float64)
        x, in_box = encode(P, ints)
        mean, spread = self.predict_features(torch.as_tensor(x, device="cuda"))
        y = mean.cpu().numpy().astype(np.float64)
        self.last_spread = spread.cpu().numpy()
        ok = in_box & ((self.last_spread <= self.config.disagreement_tol) | (not gate_disagreement))
        prices = self.to_price(y, P, ints)
        fb = ~ok
        if np.any(fb):
            prices[fb] = self.fpe_prices(P[fb], np.asarray(ints)[fb])
        return prices, fb

    def save(self, path: str) -> None:
        """Parameters of every member and the target standardisation (npz)."""
        c = self.config
        np.savez(path, mu=self.mu, sd=self.sd, hidden=c.hidden, layers=c.layers,
                 members=np.stack([m.get_params() for m in self.members]))

    def load(self, path: str) -> None:
        d = np.load(path)
        if int(d["hidden"]) != self.config.hidden or int(d["layers"]) != self.config.layers or \
                len(d["members"]) != len(self.members):
            raise ValueError("saved surrogate does not match this configuration")
        for m, th in zip(self.members, d["members"]):
            m.set_params(th)
        self.mu, self.sd = float(d["mu"]), float(d["sd"])

    def close(self):
        for m in self.members:
            m.close()
