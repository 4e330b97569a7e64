"""The autotuner on the GPU: it times the candidate shapes of a grid class,
installs the fastest, and a plan with automatic shape options then prices
exactly as the same shape chosen explicitly.  The stage-buffer count is a pure
scheduling choice (prices identical to 1e-12); the block size changes the
elimination order of the FP32 factors, so its prices agree to the
mixed-precision tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _opts(fpe, **kw):
    base = dict(disc=1, precision=1, rtol=1e-6, atol=1e-8, complex_solve=2, radau_constants=2)
    base.update(kw)
    return fpe.BatchOptions(**base)


def _restore_default(autotune):
    autotune.clear()
    autotune._loaded_default = False
    autotune.load_default()


def test_tuned_shape_is_used_by_auto_plans(engine):
    from fpe_option_b200 import autotune

    fpe = engine
    try:
        autotune.clear()
        rows = autotune.tune([(24, 16)], _opts(fpe), n_contracts=8, reps=1)
        best = (rows[0]["block_split"], rows[0]["sweep_buffers"])
        assert autotune.get_shape(1, 24, 16, 1, 2) == best
        assert len(rows[0]["ms"]) == len(autotune.CANDIDATES)
        P, I = autotune.class_batch(24, 16, 6, seed=5)
        p_auto, s_auto = fpe.price_batch(P, I, _opts(fpe))
        p_expl, s_expl = fpe.price_batch(P, I, _opts(fpe, block_split=best[0], sweep_buffers=best[1]))
        assert (s_auto == 0).all() and (s_expl == 0).all()
        np.testing.assert_allclose(p_auto, p_expl, rtol=1e-12, atol=0.0)
    finally:
        _restore_default(autotune)


@pytest.mark.parametrize("block_split", [1, 2])
def test_stage_buffers_do_not_change_prices(engine, block_split):
    from fpe_option_b200 import autotune

    fpe = engine
    P, I = autotune.class_batch(48, 24, 6, seed=9)
    ref, st = fpe.price_batch(P, I, _opts(fpe, block_split=block_split, sweep_buffers=2))
    assert (st == 0).all()
    for sb in (3, 4):
        p, st = fpe.price_batch(P, I, _opts(fpe, block_split=block_split, sweep_buffers=sb))
        assert (st == 0).all()
        np.testing.assert_allclose(p, ref, rtol=1e-12, atol=0.0)


def test_block_sizes_agree_to_the_mixed_tolerance(engine):
    from fpe_option_b200 import autotune

    fpe = engine
    P, I = autotune.class_batch(64, 32, 6, seed=4)
    p1, s1 = fpe.price_batch(P, I, _opts(fpe, block_split=1))
    p2, s2 = fpe.price_batch(P, I, _opts(fpe, block_split=2))
    assert (s1 == 0).all() and (s2 == 0).all()
    rel = np.abs(p1 - p2) / np.maximum(np.abs(p1), 1e-4)
    assert rel.max() < 1e-5, rel
