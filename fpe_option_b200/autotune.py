"""Autotuner of the Radau kernel's solve shape per grid class.

Two shape choices change how a solve uses its SM, not what it computes:

- the stage-LU block size: nv x nv blocks with three off-diagonal blocks a
  side, or (nv / 2) x (nv / 2) blocks with seven (the same band and flops;
  smaller blocks shorten each pivot inverse and halve the factorization
  scratch, larger ones take half the sequential block rows);
- the stage buffers of the staged block solves (2 to 4: each bulk copy of
  factor blocks gets one to three stage times to land).

For each grid class (discretization, n_s, n_v, factor precision, complex
stage mode) `tune` prices one seeded batch of that class per candidate shape
on the device, times the Radau kernel with CUDA events (`Plan.kernel_times`),
keeps the fastest and installs it in the engine (`fpe_tune_set`), where plans
whose block_split / sweep_buffers options are 0 look it up.  `save` / `load`
persist the table as text (one class per line), the format the engine also
reads from the file named by FPE_TUNE_TABLE; `load_default` installs the
table measured on a B200 that ships with the package.
"""
from __future__ import annotations

import os
import time

import numpy as np

from . import _lib

_HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_TABLE = os.path.join(_HERE, "tuning_b200.txt")

# (block_split, sweep_buffers)
CANDIDATES = ((1, 2), (1, 3), (1, 4), (2, 2), (2, 3), (2, 4))

# The grid classes of the batched European workload and of the knock-in workload.
BATCH_CLASSES = tuple((ns, nv) for ns in (32, 48, 64) for nv in (16, 24, 32))
BARRIER_CLASSES = tuple((ns, nv) for ns in (48, 64, 96) for nv in (24, 32, 48))

_loaded_default = False


def class_batch(n_s: int, n_v: int, n: int, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """n seeded Heston contracts of one grid class (the batched workload's
    parameter ranges, calls and puts alternating), as (params, ints) tables."""
    rng = np.random.default_rng(seed)
    P = np.zeros((n, 12))
    I = np.zeros((n, 3), np.int32)
    for j in range(n):
        P[j] = [rng.uniform(0.5, 3), rng.uniform(0.02, 0.15), rng.uniform(0.1, 0.8), rng.uniform(-0.9, 0),
                rng.uniform(0, 0.05), rng.uniform(0.1, 2), 100.0, rng.uniform(0.02, 0.2),
                100.0 * rng.uniform(0.8, 1.2), 0.0, 0.0, 300.0]
        I[j] = [n_s, n_v, 8 if j % 2 == 0 else 9]
    return P, I


def radau_ms(P, I, options, reps: int = 2) -> float:
    """The Radau kernel's device time (ms) for one batch, the best of reps runs
    after one warm-up run."""
    from . import Plan, contracts_from_arrays

    arr, keep = contracts_from_arrays(P, I)
    plan = Plan(arr, options, _keep=keep)
    try:
        plan.run()
        return min(plan.kernel_times()[3] for _ in range(reps))
    finally:
        plan.close()


def choose(times: dict) -> tuple[int, int]:
    """The fastest shape; ties go to the earlier candidate (fewer changes)."""
    best = None
    for shape in CANDIDATES:
        if shape in times and (best is None or times[shape] < times[best]):
            best = shape
    return best


def tune(classes, base_options, n_contracts: int = 148, reps: int = 2, timer=None, log=None,
         install: bool = True) -> list[dict]:
    """Time every candidate shape of each (n_s, n_v) class and install the
    fastest.  base_options: the BatchOptions the class runs with (disc,
    precision, tolerances, complex stage); its block_split / sweep_buffers
    are overridden per candidate.  timer(P, I, options) -> ms replaces the
    device timing (tests)."""
    import dataclasses

    timer = timer or (lambda P, I, o: radau_ms(P, I, o, reps))
    rows = []
    for n_s, n_v in classes:
        P, I = class_batch(n_s, n_v, n_contracts, seed=1000 + 97 * n_s + n_v)
        times = {}
        for bs, sb in CANDIDATES:
            if bs == 2 and n_v % 2:
                continue
            o = dataclasses.replace(base_options, block_split=bs, sweep_buffers=sb)
            t0 = time.perf_counter()
            times[(bs, sb)] = float(timer(P, I, o))
            if log:
                log(f"tune {n_s}x{n_v} split {bs} bufs {sb}: {times[(bs, sb)]:.3f} ms "
                    f"({time.perf_counter() - t0:.1f} s)")
        best = choose(times)
        row = {"disc": base_options.disc, "n_s": n_s, "n_v": n_v, "precision": base_options.precision,
               "complex_solve": base_options.complex_solve, "block_split": best[0], "sweep_buffers": best[1],
               "ms": {f"{k[0]},{k[1]}": v for k, v in times.items()}}
        rows.append(row)
        if install:
            set_shape(row)
    return rows


def set_shape(row: dict) -> None:
    rc = _lib.load().fpe_tune_set(row["disc"], row["n_s"], row["n_v"], row["precision"], row["complex_solve"],
                                  row["block_split"], row["sweep_buffers"])
    if rc != 0:
        raise ValueError(f"fpe_tune_set rejected {row}")


def get_shape(disc, n_s, n_v, precision, complex_solve):
    """The installed (block_split, sweep_buffers) of a class, or None."""
    import ctypes as C

    bs, sb = C.c_int32(), C.c_int32()
    if _lib.load().fpe_tune_get(disc, n_s, n_v, precision, complex_solve, C.byref(bs), C.byref(sb)) != 1:
        return None
    return bs.value, sb.value


def save(rows, path: str) -> None:
    """One class per line: disc n_s n_v precision complex_solve block_split
    sweep_buffers, then the candidates' times as a comment."""
    with open(path, "w") as f:
        f.write("# disc n_s n_v precision complex_solve block_split sweep_buffers  # Radau ms per "
                "candidate (block_split,sweep_buffers)\n")
        for r in rows:
            ms = " ".join(f"{k}={v:.3f}" for k, v in r.get("ms", {}).items())
            f.write(f"{r['disc']} {r['n_s']} {r['n_v']} {r['precision']} {r['complex_solve']} "
                    f"{r['block_split']} {r['sweep_buffers']}  # {ms}\n")


def parse(path: str) -> list[dict]:
    rows = []
    with open(path) as f:
        for line in f:
            body = line.split("#", 1)[0].split()
            if len(body) != 7:
                continue
            v = [int(x) for x in body]
            rows.append({"disc": v[0], "n_s": v[1], "n_v": v[2], "precision": v[3], "complex_solve": v[4],
                         "block_split": v[5], "sweep_buffers": v[6]})
    return rows


def load(path: str) -> int:
    """Install a saved table; returns the number of classes."""
    rows = parse(path)
    for r in rows:
        set_shape(r)
    return len(rows)


def load_default() -> int:
    """Install the B200 table shipped with the package (once per process)."""
    global _loaded_default
    if _loaded_default or not os.path.exists(DEFAULT_TABLE):
        return 0
    _loaded_default = True
    return load(DEFAULT_TABLE)


def clear() -> None:
    global _loaded_default
    _lib.load().fpe_tune_clear()
    _loaded_default = True  # an explicit clear is not undone by the default table


def main() -> None:
    """Tune the grid classes of the batched and knock-in workloads (config
    discretization, FP32 factors, direct complex stage, rtol 1e-6) on the
    current GPU and write the package's default table."""
    import argparse
    import sys

    from . import BatchOptions, build

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--contracts", type=int, default=148, help="contracts per class batch (one per SM)")
    ap.add_argument("--reps", type=int, default=2)
    args = ap.parse_args()
    build.build_library()
    base = BatchOptions(disc=1, precision=1, rtol=1e-6, atol=1e-8, complex_solve=2, radau_constants=2)
    clear()
    classes = sorted(set(BATCH_CLASSES) | set(BARRIER_CLASSES))
    rows = tune(classes, base, n_contracts=args.contracts, reps=args.reps,
                log=lambda m: print(m, file=sys.stderr, flush=True))
    save(rows, args.out)
    for r in rows:
        print(f"{r['n_s']}x{r['n_v']}: block_split {r['block_split']}, sweep_buffers {r['sweep_buffers']}")


if __name__ == "__main__":
    main()
