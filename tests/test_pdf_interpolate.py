"""Interpolation of a tabulated terminal density (reference
src/server/interpolator.mojo:14-198): Catmull-Rom bicubic on the 4 x 4
neighbourhood of the enclosing cell, indices clamped at the edges, local
coordinates clamped to [0, 1], bilinear below 4 points per axis.

CPU: the oracle restatement against properties of the rule.  It reproduces the
grid values at the nodes.  Catmull-Rom weights sum to 1 and reproduce linear
data exactly inside a uniform grid.  Points outside the grid take the edge
cell's value at t = 0 or 1.  GPU: the device kernel (binary interval search)
against the oracle (the reference's linear scan) on a Compute density, with
nodes, interior points, points outside the grid and a NaN; and the bilinear
rule on a 3 x 3 grid.  Both evaluate the same products in the same order;
FMA contraction on the device leaves ulp-level differences, so the tolerance
is 1e-13 relative to the density's scale.
"""
import numpy as np
import pytest


def test_oracle_interpolation_properties(oracle):
    rng = np.random.default_rng(1)
    sp = np.sort(rng.uniform(0, 10, 12))
    vp = np.sort(rng.uniform(0, 1, 9))
    pdf = rng.standard_normal((12, 9))
    # nodes (interior cells: t = 0 picks weight 1 on the node)
    S, V = np.meshgrid(sp[:-1], vp[:-1], indexing="ij")
    got = oracle.pdf_interpolate(sp, vp, pdf, S.ravel(), V.ravel())
    np.testing.assert_allclose(got, pdf[:-1, :-1].ravel(), rtol=0, atol=1e-14)
    # linear data on a uniform grid, away from the clamped edge cells
    us, uv = np.linspace(0, 4, 9), np.linspace(0, 1, 6)
    lin = 2.0 + 3.0 * us[:, None] - 1.5 * uv[None, :]
    qs, qv = rng.uniform(us[1], us[-2], 50), rng.uniform(uv[1], uv[-2], 50)
    np.testing.assert_allclose(oracle.pdf_interpolate(us, uv, lin, qs, qv), 2.0 + 3.0 * qs - 1.5 * qv,
                               rtol=0, atol=1e-12)
    # outside the grid: clamped to the edge cells
    out = oracle.pdf_interpolate(us, uv, lin, [-5.0, 99.0], [0.5, 0.5])
    edge = oracle.pdf_interpolate(us, uv, lin, [us[0], us[-1] - 1e-300], [0.5, 0.5])
    np.testing.assert_allclose(out, [edge[0], 2.0 + 3.0 * us[-1] - 1.5 * 0.5], atol=1e-12)
    # bilinear below 4 points per axis
    bs, bv = np.array([0.0, 1.0, 3.0]), np.array([0.0, 2.0, 4.0])
    bl = 1.0 + bs[:, None] * 2.0 + bv[None, :] * 0.5 + bs[:, None] * bv[None, :]
    q = oracle.pdf_interpolate(bs, bv, bl, [0.5, 2.0], [1.0, 3.0])
    np.testing.assert_allclose(q, [1.0 + 1.0 + 0.5 + 0.5, 1.0 + 4.0 + 1.5 + 6.0], atol=1e-12)


@pytest.mark.gpu
def test_device_interpolation_matches_oracle(engine, oracle):
    fpe = engine
    c = fpe.Compute(S0=60.0, V0=0.1, T=0.6, r=0.1, n_s=12, n_v=12, option_type="european_call",
                    s_max=150.0, num_insert=30)
    g, pdf = c.grid_points, c.pdf
    rng = np.random.default_rng(4)
    n = 4096
    s = rng.uniform(g.s[0] - 5.0, g.s[-1] + 5.0, n)
    v = rng.uniform(g.v[0] - 0.1, g.v[-1] + 0.1, n)
    s[:20], v[:20] = g.s[3:23], g.v[5:25]   # nodes
    s[20], v[20] = np.nan, 0.5
    got = c.pdf_interpolate(s, v)
    ref = oracle.pdf_interpolate(g.s, g.v, pdf, s, v)
    scale = np.max(np.abs(pdf))
    ok = np.isfinite(ref)
    np.testing.assert_allclose(got[ok], ref[ok], rtol=0, atol=1e-13 * scale)
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    np.testing.assert_allclose(got[:20], pdf[3:23, 5:25].diagonal(), rtol=0, atol=1e-13 * scale)
    # bilinear rule on a 3 x 3 grid
    bs, bv = np.array([0.0, 1.0, 3.0]), np.array([0.0, 2.0, 4.0])
    bl = rng.standard_normal((3, 3))
    qs, qv = rng.uniform(-1, 4, 64), rng.uniform(-1, 5, 64)
    np.testing.assert_allclose(fpe.interpolate_pdf(bs, bv, bl, qs, qv), oracle.pdf_interpolate(bs, bv, bl, qs, qv),
                               rtol=0, atol=1e-14)
