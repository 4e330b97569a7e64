"""The autotuner's table logic on the CPU: candidate choice, the text format
the engine also reads, and install / look-up through the C ABI (host-side
state only; no kernel runs)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def tuner():
    from fpe_option_b200 import _lib, autotune, build

    build.build_library()
    _lib.load()
    return autotune


def test_choose_takes_the_fastest_and_breaks_ties_in_candidate_order(tuner):
    t = {(1, 2): 3.0, (1, 3): 2.0, (2, 2): 2.0, (2, 3): 5.0}
    assert tuner.choose(t) == (1, 3)
    assert tuner.choose({(2, 4): 1.0}) == (2, 4)


def test_tune_with_a_fake_timer_installs_and_round_trips(tuner, tmp_path):
    import fpe_option_b200 as fpe

    base = fpe.BatchOptions(disc=1, precision=1, complex_solve=2)
    # a timer that prefers half-width blocks on wide grids and 3 buffers otherwise
    def timer(P, I, o):
        nv = int(I[0, 1])
        assert len(P) == 4 and (I[:, 0] == I[0, 0]).all()
        return (1.0 if (o.block_split == 2) == (nv >= 48) else 2.0) + (0.0 if o.sweep_buffers == 3 else 0.5)

    tuner.clear()
    rows = tuner.tune([(32, 16), (96, 48), (20, 15)], base, n_contracts=4, timer=timer)
    assert [(r["block_split"], r["sweep_buffers"]) for r in rows] == [(1, 3), (2, 3), (1, 3)]
    assert "2,2" not in rows[2]["ms"]  # odd n_v: no half-width blocks
    assert tuner.get_shape(1, 96, 48, 1, 2) == (2, 3)
    assert tuner.get_shape(1, 96, 48, 0, 2) is None  # another precision is another class
    path = str(tmp_path / "table.txt")
    tuner.save(rows, path)
    tuner.clear()
    assert tuner.get_shape(1, 32, 16, 1, 2) is None
    assert tuner.load(path) == 3
    assert tuner.get_shape(1, 32, 16, 1, 2) == (1, 3)
    assert [(r["n_s"], r["n_v"]) for r in tuner.parse(path)] == [(32, 16), (96, 48), (20, 15)]
    tuner.clear()


def test_bad_shapes_are_rejected(tuner):
    from fpe_option_b200 import _lib

    L = _lib.load()
    assert L.fpe_tune_set(1, 32, 16, 1, 2, 3, 2) < 0
    assert L.fpe_tune_set(1, 32, 16, 1, 2, 1, 5) < 0
    assert L.fpe_tune_set(1, 32, 16, 1, 2, 1, 0) == 0
    tuner.clear()


def test_class_batch_is_seeded_and_of_one_class(tuner):
    P, I = tuner.class_batch(48, 24, 6, seed=3)
    P2, _ = tuner.class_batch(48, 24, 6, seed=3)
    assert np.array_equal(P, P2)
    assert (I[:, 0] == 48).all() and (I[:, 1] == 24).all() and set(I[:, 2]) == {8, 9}


def test_shipped_table_covers_both_workloads():
    """The B200 table in the package names every grid class of the batched and
    knock-in workloads once (config discretization, FP32 factors, direct
    complex stage), with a valid shape; half-width blocks exactly where nv x nv
    scratch would not fit shared memory (n_v = 48)."""
    from fpe_option_b200 import autotune

    rows = autotune.parse(autotune.DEFAULT_TABLE)
    keys = [(r["n_s"], r["n_v"]) for r in rows]
    assert sorted(keys) == sorted(set(autotune.BATCH_CLASSES) | set(autotune.BARRIER_CLASSES))
    for r in rows:
        assert (r["disc"], r["precision"], r["complex_solve"]) == (1, 1, 2)
        assert (r["block_split"], r["sweep_buffers"]) in autotune.CANDIDATES
        assert r["block_split"] == (2 if r["n_v"] == 48 else 1), r
