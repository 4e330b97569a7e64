"""CPU checks of the surrogate's oracle: BF16 rounding, and the analytic
gradient against central finite differences of the unrounded network."""
import numpy as np

from oracle import mlp_oracle as mo


def _params(layout, rng):
    n_in, in_pad, hidden, layers = layout
    parts = []
    for l in range(layers):
        fin = in_pad if l == 0 else hidden
        W = rng.uniform(-1, 1, (hidden, fin)) / np.sqrt(fin)
        if l == 0:
            W[:, n_in:] = 0.0
        parts += [W.ravel(), rng.uniform(-0.1, 0.1, hidden)]
    parts += [rng.uniform(-1, 1, hidden) / np.sqrt(hidden), [0.05]]
    return np.concatenate(parts).astype(np.float32)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 0.0, 3.0e38], np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0  # tie -> even mantissa
    assert r[2] == 1.0 + 4 * 2 ** -8  # tie -> even (up)
    assert r[3] == 1.0
    assert r[4] == -2.5 and r[5] == 0.0
    # every result is representable in 8 mantissa bits
    m = r[np.isfinite(r) & (r != 0)]
    assert np.all(np.frexp(m)[0] * 256 == np.round(np.frexp(m)[0] * 256))


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    layout = (5, 16, 8, 2)
    theta = _params(layout, rng).astype(np.float64)
    x = rng.uniform(-1, 1, (7, 5))
    t = rng.uniform(0, 1, 7)
    w = rng.uniform(0.5, 2, 7)
    loss, g = mo.gradient(theta, layout, x, t, w, exact=True)
    idx = rng.choice(np.flatnonzero(g != 0), 40, replace=False)
    for i in idx:
        e = np.zeros_like(theta)
        e[i] = 1e-6
        lp, _ = mo.gradient(theta + e, layout, x, t, w, exact=True)
        lm, _ = mo.gradient(theta - e, layout, x, t, w, exact=True)
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_adam_step_rule():
    # reference src/nn/adam.mojo:31-64: bias-corrected moments, eps outside the root
    th, m, v = mo.adam_step(np.array([1.0]), np.array([0.5]), np.zeros(1), np.zeros(1), 1, 0.1)
    assert np.allclose(th, 1.0 - 0.1 * 0.5 / (0.5 + 1e-8))
    assert np.allclose(m, 0.05) and np.allclose(v, 0.00025)
