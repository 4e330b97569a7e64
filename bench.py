"""Benchmark: FPE option prices/sec on B200 (batched, mixed precision).

Workload (one "step" = pricing one batch): 256 European Heston contracts drawn
from a fixed seed with kappa~U[0.5,3], theta~U[0.02,0.15], eta~U[0.1,0.8],
rho~U[-0.9,0], V0~U[0.02,0.2], r~U[0,0.05], T~U[0.1,2], S0=100,
K/S0~U[0.8,1.2], calls/puts 50/50, grids n_s in {32,48,64} x n_v in {16,24,32}
(sinh-stretched clamped cubic B-splines, s_max = 3 S0, v_max = 1), solved in
one launch sequence with FP32 stage factors + FP64 Newton residuals, direct
complex stage solve and exact Radau IIA constants.  Synthetic data (no public
dataset is involved).  With N GPUs (one process each) the seeded batch has
256 N contracts, split across the ranks by estimated solve cost; each rank
prices its shard and one all-gather returns the whole price vector (weak
scaling: the work per GPU stays fixed as N grows).

value: prices/s with the contract descriptors resident in HBM, device time
of the five kernels (CUDA events on the launching stream), max over ranks.
e2e:   prices/s through the public C ABI from host contracts to host prices
(plan creation with its host-to-device copy, kernels, device-to-host copy).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FPE option prices/sec on 1 B200 at <=1e-4 rel err: batched vs plain vs surrogate"
N_CONTRACTS = 256
RTOL = 1e-6  # Radau tolerance of the batched run (atol = rtol * 1e-2)
REF_RTOL = 1e-10  # FP64 reference run used to state the error


def make_batch(n: int, seed: int):
    """Seeded Heston contract draws: (n, 12) float + (n, 3) int tables."""
    rng = np.random.default_rng(seed)
    P = np.zeros((n, 12))
    I = np.zeros((n, 3), np.int32)
    for j in range(n):
        P[j] = [rng.uniform(0.5, 3), rng.uniform(0.02, 0.15), rng.uniform(0.1, 0.8),
                rng.uniform(-0.9, 0), rng.uniform(0, 0.05), rng.uniform(0.1, 2), 100.0,
                rng.uniform(0.02, 0.2), 100.0 * rng.uniform(0.8, 1.2), 0.0, 0.0, 300.0]
        I[j] = [rng.choice([32, 48, 64]), rng.choice([16, 24, 32]), 8 if j % 2 == 0 else 9]
    return P, I


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def load_traffic():
    """Per-launch DRAM bytes of k_radau from the committed ncu summary (or None)."""
    path = os.path.join(ROOT, "profiles", "k_radau_traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device),
                                      f"--query-gpu={self.Q}", "--format=csv,noheader,nounits"],
                                     capture_output=True, text=True, timeout=5).stdout
                for line in out.strip().splitlines():
                    self.rows.append([c.strip() for c in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) > 8:
                for k, nm in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def class_sample(I, per_class: int = 2):
    """The first `per_class` contracts of each (n_s, n_v) grid class of a
    batched-workload table, in batch order (the oracle-checked sample)."""
    idx = []
    for ns in (32, 48, 64):
        for nv in (16, 24, 32):
            idx += list(np.flatnonzero((I[:, 0] == ns) & (I[:, 1] == nv))[:per_class])
    return np.array(sorted(idx), dtype=np.int64)


def max_over_ranks(x: float, dist, world: int, device) -> float:
    """The slowest rank's time (every rank takes the same collective step)."""
    if world <= 1:
        return x
    import torch

    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, per_rank: int, steps: int, seconds: float) -> float:
    """Whole-job rate: the units all ranks processed over the slowest rank's time."""
    return world * per_rank * steps / seconds


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# FP32 CUDA-core peak of a B200 (nominal): 148 SMs x 128 FP32 lanes x 2 flops
# per FMA x 1.965 GHz.
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def factorization_flops(ns: int, nv: int) -> float:
    """Flops of one real + one complex stage factorization of the block-banded
    LU (nv x nv blocks, 3 off-diagonal blocks a side): per block row with nr
    off-diagonal blocks, (1 + nr)^2 block products of 2 nv^3 flops (the
    pivot inverse, nr L and nr W products, nr^2 Schur updates), and 4x that
    for the complex system.  Half-width blocks hold the same band and cost
    the same within the band's edges."""
    rows = sum((1 + min(3, ns - 1 - i)) ** 2 for i in range(ns))
    return 5.0 * 2.0 * nv ** 3 * rows


def factorization_roofline(sinfo, radau_ms: float) -> dict:
    """The stage factorizations' FP32 CUDA-core rate: their algorithmic flops
    (factorization_flops x factorizations, per solve) over the Radau kernel's
    time, and over the SM time the factorizations themselves took (the
    per-solve phase timers, summed over solves and spread over the 148 SMs)."""
    flops = float(sum(int(r[13]) * factorization_flops(int(r[7]), int(r[8])) for r in sinfo if r[7] > 0))
    fac_share = float(sinfo[:, 18].sum()) / max(1.0, float(sinfo[:, 21].sum()))
    ach = flops / (radau_ms / 1000.0) / 1e12
    in_fac = ach / max(fac_share, 1e-9)
    return {"bound": "fp32_fma", "kernel": "k_radau (stage factorizations)", "achieved": ach,
            "peak": FP32_PEAK_TFLOPS, "unit": "TFLOP/s", "frac": ach / FP32_PEAK_TFLOPS,
            "peak_kind": "nominal (148 SMs x 128 FP32 lanes x 2 x 1.965 GHz)",
            "algorithmic_flops": flops, "factorization_share_of_kernel": fac_share,
            "achieved_during_factorization": in_fac, "frac_during_factorization": in_fac / FP32_PEAK_TFLOPS}


def cpu_baseline_run(P, I, rtol, n_threads, idx=None):
    """The oracle port on the contracts idx (all when None): one solve per
    thread, solves spread over n_threads host threads, the same discretization
    and Radau tolerance as the GPU arm, and the reference's own complex stage
    algorithm (GMRES(10) preconditioned by the real stage factors).  Returns
    (prices/s, seconds, prices)."""
    from oracle import pyoracle as po

    opt = po.options(disc=1, rtol=rtol, atol=rtol * 1e-2, radau_constants=2)
    idx = np.arange(len(P)) if idx is None else np.asarray(idx)
    t = time.perf_counter()
    prices = po.price_batch(P[idx], I[idx], opt, n_threads=n_threads)
    dt = time.perf_counter() - t
    return len(idx) / dt, dt, prices


def run_reference_arm(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    nc = args.contracts
    P, I = make_batch(nc, args.seed)
    cores = os.cpu_count() or 1
    sample = max(cores, min(args.cpu_sample, nc))
    rates = []
    for _ in range(args.warmup):
        cpu_baseline_run(P, I, args.rtol, cores, np.arange(min(sample, cores)))
    for s in range(args.steps):
        sl = (np.arange(sample) + s * sample) % nc
        r, _, _ = cpu_baseline_run(P, I, args.rtol, cores, sl)
        rates.append(r)
    v = float(np.mean(rates))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "prices/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * sample / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{args.contracts} European Heston contracts, mixed grids 32-64 x 16-32",
                       "rtol": args.rtol, "contracts_per_step": sample},
            "cpu_baseline": {"value": v, "unit": "prices/s", "cores": cores, "kind": "port",
                             "sample": f"{sample} contracts of the bench batch per step, "
                                       f"oracle C++ FP64 restatement, {cores} threads"},
            "e2e": {"value": v, "unit": "prices/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--contracts", type=int, default=N_CONTRACTS,
                    help="contracts per GPU per step (smaller batches serve profiling)")
    ap.add_argument("--rtol", type=float, default=RTOL)
    ap.add_argument("--precision", type=int, default=1)
    ap.add_argument("--cpu-sample", type=int, default=18,
                    help="CPU-baseline contracts (spread evenly over the nine grid classes)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-surrogate-rate", dest="surrogate_rate", action="store_false",
                    help="skip the surrogate inference rate in the batch line")
    ap.add_argument("--no-cf-check", dest="cf_check", action="store_false",
                    help="skip the characteristic-function check and rate in the batch line")
    ap.add_argument("--no-barrier", dest="barrier", action="store_false",
                    help="skip the knock-in workload's compact summary in the batch line")
    ap.add_argument("--plain-sample", type=int, default=9,
                    help="contracts timed on the plain one-solve-per-launch FP64 path (one per grid class first)")
    ap.add_argument("--workload", default="batch",
                    choices=["batch", "barrier", "surrogate", "calibration", "layer"],
                    help="batch: the batched FPE pricing line (default); surrogate / calibration: "
                         "the learned part's measurements; layer: the surrogate network's forward alone "
                         "(65,536 rows, random weights), the case its product kernel is profiled on")
    ap.add_argument("--train", type=int, default=65536, help="surrogate training prices")
    ap.add_argument("--surfaces", type=int, default=5, help="calibration: seeded surfaces")
    ap.add_argument("--surrogate-file", default=None,
                    help="calibration: load a trained European ensemble (npz) instead of training; "
                         "if the file does not exist, train and save it there")
    ap.add_argument("--epochs", type=int, default=None,
                    help="surrogate epochs (default 200 for --workload surrogate, 2000 for calibration)")
    ap.add_argument("--batch", type=int, default=None,
                    help="surrogate batch (default 4096 for --workload surrogate, 1024 for calibration)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "barrier":
        return run_barrier_workload(args)
    if args.workload == "layer":
        return run_layer_workload(args)
    if args.workload != "batch":
        return run_learned_workload(args)

    import torch
    import torch.distributed as dist

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from fpe_option_b200 import build

    if rank == 0:
        build.build_library()
    if world > 1:
        dist.barrier()
    import fpe_option_b200 as fpe

    if not fpe.is_available():
        raise RuntimeError("CUDA engine unavailable")
    from fpe_option_b200 import sharding

    n_total = args.contracts * world  # weak scaling: a fixed share per GPU
    P_all, I_all = make_batch(n_total, args.seed)
    shards = sharding.partition(sharding.solve_costs(P_all, I_all), world)
    mine = shards[rank]
    P, I = P_all[mine], I_all[mine]
    nc = len(mine)
    opts = fpe.BatchOptions(disc=1, precision=args.precision, rtol=args.rtol,
                            atol=args.rtol * 1e-2, complex_solve=2, radau_constants=2)
    arr, keep = fpe.contracts_from_arrays(P, I)
    plan = fpe.Plan(arr, opts, _keep=keep)
    # a dedicated (non-default) stream: the kernels and the timing events share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream
    assert sptr != 0
    # accuracy: the same batch in FP64 at a tight tolerance (untimed)
    ref = fpe.Plan(arr, fpe.BatchOptions(disc=1, precision=0, rtol=REF_RTOL,
                                         atol=REF_RTOL * 1e-2, complex_solve=2,
                                         radau_constants=2), _keep=keep)
    ref.run()
    p_ref, _, _, _, st_ref = ref.results()
    ref.close()
    for _ in range(max(args.warmup, 3)):
        plan.run(sptr)
    torch.cuda.synchronize()
    p_out, _, _, _, st = plan.results()
    floor = 1e-6 * 100.0
    rel = np.abs(p_out - p_ref) / np.maximum(np.abs(p_ref), floor)
    rel_unfloored = np.abs(p_out - p_ref) / np.abs(p_ref)
    # per-kernel times and the roofline of the dominant kernel (k_radau)
    ktimes = plan.kernel_times(sptr)
    stats = plan.stats()
    sinfo = plan.solve_info()
    # ---- device-resident timed region ------------------------------------------
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_launch = 0
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            n_launch += plan.run(sptr)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, world, "cuda")
    if world > 1:
        dist.barrier()
    value = n_total * args.steps / (ms / 1000.0)
    # the whole batch's prices on every rank (one all-gather; untimed here)
    p_all, st_all = sharding.gather_prices(p_out, st, shards, dist, "cuda") if world > 1 else (p_out, st)
    # ---- end to end through the public C ABI (host contracts -> host prices) -----
    pinned = torch.empty((nc, 12), dtype=torch.float64).pin_memory()
    pinned.copy_(torch.from_numpy(P))
    Ph = pinned.numpy()
    h2d = nc * (C_SIZE_CONTRACT()) + nc * 8
    d2h = nc * 8 + stats["solves"] * 80
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        a2, k2 = fpe.contracts_from_arrays(Ph, I)
        pl = fpe.Plan(a2, opts, _keep=k2)
        pl.run(sptr)
        pe, _, _, _, se = pl.results()
        pl.close()
        if world > 1:  # every rank ends the step with the whole batch's prices
            sharding.gather_prices(pe, se, shards, dist, "cuda")
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, world, "cuda")
    e2e = n_total * args.steps / e2e_s
    # ---- roofline of k_radau -----------------------------------------------------
    peak, peak_kind = load_peaks()
    radau_ms = ktimes[3]
    achieved = stats["factor_bytes"] / (radau_ms / 1000.0) / 1e9
    traffic = load_traffic()
    fp32 = factorization_roofline(sinfo, radau_ms)
    # ---- CPU baseline (oracle port), rank 0, bounded sample -------------------------
    # The sample is two contracts of each of the nine grid classes; its oracle
    # prices also give this run's error against the FP64 oracle.
    cpu = None
    oracle_err = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        sidx = class_sample(I, max(1, args.cpu_sample // 9))
        rate, dt, p_orc = cpu_baseline_run(P, I, args.rtol, cores, sidx)
        cpu = {"value": rate, "unit": "prices/s", "cores": cores, "kind": "port",
               "sample": f"{len(sidx)} contracts of the same batch ({len(sidx) // 9} per grid class), oracle C++ "
                         f"FP64 restatement on {cores} host threads, {dt:.1f} s"}
        e_orc = np.abs(p_out[sidx] - p_orc) / np.maximum(np.abs(p_orc), floor)
        p64, _ = fpe.price_batch(P[sidx], I[sidx], fpe.BatchOptions(
            disc=1, precision=0, rtol=args.rtol, atol=args.rtol * 1e-2, complex_solve=2, radau_constants=2))
        e64 = np.abs(p64 - p_orc) / np.maximum(np.abs(p_orc), floor)
        oracle_err = {"max_rel_err_vs_oracle": float(e_orc.max()), "median_rel_err_vs_oracle": float(np.median(e_orc)),
                      "contracts": int(len(sidx)), "err_floor": floor,
                      "fp64_max_rel_err_vs_oracle": float(e64.max()),
                      "note": "this run's mixed-precision prices against the oracle's FP64 prices at the same rtol, "
                              "on the CPU-baseline sample (every grid class); fp64_...: the GPU's FP64-factor "
                              "path on the same sample and rtol"}
    # ---- surrogate inference rate (3-member BF16 tensor-core ensemble) ---------------
    sur = None
    if rank == 0 and world == 1 and args.surrogate_rate:
        from fpe_option_b200.surrogate import SurrogateConfig, SurrogatePricer, draw_contracts, encode

        pr = SurrogatePricer(SurrogateConfig(members=3))
        Q, J = draw_contracts(1 << 20, seed=7, kind="mixed", grid=(48, 24))
        xq = torch.as_tensor(encode(Q, J)[0], device="cuda")
        for _ in range(3):
            pr.predict_features(xq)
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        for _ in range(5):
            pr.predict_features(xq)
        s1.record()
        torch.cuda.synchronize()
        sms = s0.elapsed_time(s1) / 5
        sur = {"value": (1 << 20) / (sms / 1000.0), "unit": "prices/s", "queries": 1 << 20,
               "note": "inference of the 3-member ensemble (untrained weights: the rate does not depend on "
                       "them); trained accuracy: bench.py --workload surrogate / calibration"}
        pr.close()
    # ---- closed form: Heston characteristic-function prices of the same Europeans -----
    cfb = None
    if rank == 0 and world == 1 and args.cf_check:
        from fpe_option_b200 import _lib

        cf, cst = fpe.heston_cf_price(P, I)
        ok = cst == 0
        dev = np.abs(p_ref - cf)[ok] / np.maximum(np.abs(cf[ok]), 1e-3 * 100.0)
        # the closed-form kernel's own rate on 2^18 device-resident prices
        nq = 1 << 18
        rep = np.resize(np.arange(nc), nq)
        qP = torch.as_tensor(np.ascontiguousarray(P[rep][:, :8]), device="cuda")
        qK = torch.as_tensor(np.ascontiguousarray(P[rep][:, 8]), device="cuda")
        qput = torch.as_tensor((I[rep, 2] == 9).astype(np.int32), device="cuda")
        qout = torch.empty(nq, dtype=torch.float64, device="cuda")
        L = _lib.load()
        for _ in range(3):
            L.fpe_heston_cf_batch(qP.data_ptr(), qK.data_ptr(), qput.data_ptr(), nq, qout.data_ptr(), sptr)
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        for _ in range(3):
            L.fpe_heston_cf_batch(qP.data_ptr(), qK.data_ptr(), qput.data_ptr(), nq, qout.data_ptr(), sptr)
        c1.record(stream)
        torch.cuda.synchronize()
        cms = c0.elapsed_time(c1) / 3
        # the error grows as the Feller ratio 2 kappa theta / sigma^2 falls: the variance
        # density becomes singular at v = 0 and the v grid cannot follow it
        feller = (2.0 * P[:, 0] * P[:, 1] / P[:, 2] ** 2)[ok]
        bins = {}
        for name, lo, hi in (("feller>=1", 1.0, np.inf), ("0.5<=feller<1", 0.5, 1.0),
                             ("feller<0.5", 0.0, 0.5)):
            m = (feller >= lo) & (feller < hi)
            if m.any():
                bins[name] = {"contracts": int(m.sum()), "median_rel_dev": float(np.median(dev[m])),
                              "max_rel_dev": float(dev[m].max())}
        cfb = {"fpe_vs_cf_median_rel_dev": float(np.median(dev)), "fpe_vs_cf_max_rel_dev": float(dev.max()),
               "contracts": int(ok.sum()), "by_feller_ratio": bins, "cf_rate": nq / (cms / 1000.0),
               "unit": "prices/s",
               "note": "discretization error of the FPE prices (the tight-tolerance FP64 run of the same "
                       "batch; floor 1e-3 S0) against the FP64 characteristic-function price; cf_rate: "
                       "k_heston_cf on 2^18 device-resident prices"}
    # ---- the knock-in workload (config 2), compact: 1 warm-up run, 1 timed run -------
    barrier = None
    if rank == 0 and world == 1 and args.barrier:
        barrier = barrier_measure(fpe, torch, stream, 1, 1, args.precision, args.rtol, args.seed)
        barrier["note"] = ("1024 knock-in contracts (2048 solves, grids 48-96 x 24-48) in one launch sequence; "
                           "one warm-up and one timed run; full measurement: bench.py --workload barrier")
    # ---- plain path: one contract per launch sequence, FP64 factors ---------------
    plain = None
    if rank == 0 and world == 1 and args.plain_sample > 0:
        popts = fpe.BatchOptions(disc=1, precision=0, rtol=args.rtol, atol=args.rtol * 1e-2,
                                 complex_solve=2, radau_constants=2)
        # one contract of each grid class (then more in batch order, up to the
        # sample size), each end to end through its own plan: host contract in,
        # host price out, the same path the batched e2e figure times
        first = list(class_sample(I, 1))
        rest = [j for j in range(nc) if j not in set(first)]
        idx = sorted((first + rest)[:args.plain_sample])
        m = len(idx)
        one = [fpe.contracts_from_arrays(P[j:j + 1], I[j:j + 1]) for j in idx]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for a1, k1 in one:
            pl = fpe.Plan(a1, popts, _keep=k1)
            pl.run(sptr)
            pl.results()
            pl.close()
        dt = time.perf_counter() - t0
        plain = {"value": m / dt, "unit": "prices/s",
                 "sample": f"{m} contracts, one of each of the nine grid classes first, each its own plan "
                           "and launch sequence end to end (host contract in, host price out), FP64 factors, "
                           "same rtol",
                 "batched_over_plain": e2e / (m / dt), "compared": "batched e2e over plain e2e"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "prices/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32-factors/f64" if args.precision == 1 else "f64", "data": "synthetic",
            "config": {"workload": f"{nc} European Heston contracts per GPU, mixed grids "
                                   "32-64 x 16-32, one launch sequence",
                       "rtol": args.rtol, "atol": args.rtol * 1e-2, "precision": args.precision,
                       "complex_stage": "direct block LU", "radau_constants": "exact",
                       "l2": "inputs and factors larger than L2 (126 MB)",
                       "max_rel_err_vs_fp64": float(rel.max()), "err_floor": floor,
                       "max_rel_err_unfloored": float(rel_unfloored.max()),
                       "oracle_parity": oracle_err,
                       "fp64_reference_rtol": REF_RTOL,
                       "status_ok": bool((st == 0).all() and (st_ref == 0).all())},
            "e2e": {"value": e2e, "unit": "prices/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": n_launch,
            "kernel_ms": {"setup": ktimes[0], "galerkin": ktimes[1], "ic": ktimes[2],
                          "radau": ktimes[3], "payoff": ktimes[4]},
            "solver": {k: int(v) for k, v in stats.items()},
            "roofline": {"bound": "hbm", "kernel": "k_radau", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind,
                         "traffic": traffic.get("bytes_per_launch") if traffic else None,
                         "algorithmic_bytes": int(stats["factor_bytes"])},
            "roofline_fp32_factorization": fp32,
            "barrier_knock_in": barrier,
            "cpu_baseline": cpu,
            "plain_fp64_one_per_launch": plain,
            "surrogate_inference": sur,
            "closed_form_check": cfb,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0



# ---------------------------------------------------------------------------------
# The learned part: surrogate training / inference and calibration (1 GPU)
# ---------------------------------------------------------------------------------
SUR_GRID = (48, 24)


def _fpe_options(fpe):
    return fpe.BatchOptions(disc=1, precision=1, rtol=1e-6, atol=1e-8, complex_solve=2,
                            radau_constants=2)


def _train_surrogate(args, kind, n_train, log, epochs, batch):
    """FPE training prices (timed), 90/10 split, ensemble training (timed)."""
    import torch

    import fpe_option_b200 as fpe
    from fpe_option_b200.surrogate import SurrogateConfig, SurrogatePricer, draw_contracts, encode

    pr = SurrogatePricer(SurrogateConfig(members=3, batch=batch, epochs=epochs, seed=args.seed),
                         fpe_options=_fpe_options(fpe))
    P, I = draw_contracts(n_train, seed=1000 + args.seed, kind=kind, grid=SUR_GRID)
    t0 = time.perf_counter()
    y = pr.fpe_prices(P, I)
    t_gen = time.perf_counter() - t0
    n_hold = n_train // 10
    tr, ho = slice(n_hold, None), slice(0, n_hold)
    t0 = time.perf_counter()
    losses = pr.fit(P[tr], I[tr], y[tr], log=log)
    t_fit = time.perf_counter() - t0
    x = torch.as_tensor(encode(P[ho], I[ho])[0], device="cuda")
    mean, spread = pr.predict_features(x)
    got = pr.to_price(mean.cpu().numpy(), P[ho], I[ho])
    ref = y[ho]
    floor = 0.2  # 2e-3 S0
    rel = np.abs(got - ref) / (np.abs(ref) + floor)
    held = {"n": int(n_hold), "median_rel_err": float(np.median(rel)),
            "p90_rel_err": float(np.quantile(rel, 0.9)), "max_rel_err": float(rel.max()),
            "err_floor": floor, "trusted_frac": float(np.mean(spread.cpu().numpy() <= pr.config.disagreement_tol))}
    return pr, {"train_prices": int(n_train - n_hold), "fpe_generation_s": t_gen,
                "fpe_generation_prices_per_s": n_train / t_gen, "training_s": t_fit,
                "final_losses": losses, "held_out": held}


def run_layer_workload(args):
    """The surrogate network's forward (12 -> 256 x 4 -> 1, random weights) on
    65,536 random rows: per forward, one input-layer product (K = 16), three
    65,536 x 256 x 256 layer products (the persistent TMA kernel) and the output
    layer.  Warm-up forwards first, then `steps` timed ones (CUDA events)."""
    import torch

    from fpe_option_b200 import build
    from fpe_option_b200.surrogate import Mlp

    build.build_library()
    n = 65536
    net = Mlp(n_in=12, hidden=256, layers=4, max_rows=n, seed=1 + args.seed)
    x = torch.randn(n, 12, device="cuda", generator=torch.Generator("cuda").manual_seed(args.seed))
    y = torch.empty(n, device="cuda")
    for _ in range(max(args.warmup, 3)):
        net.forward_dev(x, y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        net.forward_dev(x, y)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    flops = 2.0 * n * (16 * 256 + 3 * 256 * 256 + 256)
    print(json.dumps({"metric": "surrogate network forward, 65536 rows", "value": n / (ms / 1000.0),
                      "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3),
                      "ms_per_step": ms, "higher_is_better": True, "dtype": "bf16/f32", "data": "synthetic",
                      "workload": "layer", "tflops": flops / (ms / 1000.0) / 1e12,
                      "config": {"workload": "MLP 12-256x4-1 SiLU, random weights, 65536 random rows"}}),
          flush=True)
    net.close()
    return 0


def run_learned_workload(args):
    import torch

    import fpe_option_b200 as fpe
    from fpe_option_b200 import build

    build.build_library()
    if not fpe.is_available():
        raise RuntimeError("CUDA engine unavailable")
    log = (lambda m: print(m, file=sys.stderr, flush=True))
    if args.workload == "surrogate":
        from fpe_option_b200.surrogate import draw_contracts, encode

        ep, bs = args.epochs or 200, args.batch or 4096
        pr, info = _train_surrogate(args, "mixed", args.train, log, ep, bs)
        nq = 1 << 20
        Q, J = draw_contracts(nq, seed=7 + args.seed, kind="mixed", grid=SUR_GRID)
        x = torch.as_tensor(encode(Q, J)[0], device="cuda")
        for _ in range(max(args.warmup, 3)):
            pr.predict_features(x)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            pr.predict_features(x)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        line = {"metric": "surrogate prices/s (3-member BF16 tensor-core ensemble) and held-out error vs FPE",
                "value": nq / (ms / 1000.0), "unit": "prices/s", "n_gpus": 1, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "dtype": "bf16/f32",
                "data": "synthetic", "workload": "surrogate",
                "config": {"workload": f"{args.train} FPE prices ({SUR_GRID[0]}x{SUR_GRID[1]} grids, European "
                                       "and barrier, 90/10 split), MLP 12-256x4-1 SiLU, Adam lr 1e-3 cosine, "
                                       f"batch {bs}, {ep} epochs; inference on 1048576 random queries"},
                **info}
        print(json.dumps(line), flush=True)
        pr.close()
        return 0
    # ---- calibration: 15 strikes x 8 maturities, FPE-only vs surrogate in the loop ----
    from fpe_option_b200.calibration import Surface, calibrate_fpe, calibrate_with_surrogate, contract_tables

    ep, bs = args.epochs or 2000, args.batch or 1024
    if args.surrogate_file and os.path.exists(args.surrogate_file):
        from fpe_option_b200.surrogate import SurrogateConfig, SurrogatePricer

        pr = SurrogatePricer(SurrogateConfig(members=3, batch=bs, epochs=ep, seed=args.seed),
                             fpe_options=_fpe_options(fpe))
        pr.load(args.surrogate_file)
        info = {"loaded": args.surrogate_file}
    else:
        pr, info = _train_surrogate(args, "european", args.train, log, ep, bs)
        info["epochs"], info["batch"] = ep, bs
        if args.surrogate_file:
            pr.save(args.surrogate_file)
    surfaces = []
    kw = {"grid": SUR_GRID}
    noise = 1e-4 * 100.0
    res = {"fpe_only": [], "surrogate": [], "defect": [], "hybrid": []}
    for k in range(args.surfaces):
        rng = np.random.default_rng(4242 + 97 * k + args.seed)
        truth = np.array([rng.uniform(0.8, 2.5), rng.uniform(0.03, 0.12), rng.uniform(0.2, 0.7),
                          rng.uniform(-0.8, -0.2), rng.uniform(0.03, 0.15)])
        surf = Surface.grid(100.0, 0.02, np.linspace(0.7, 1.3, 15), np.linspace(0.1, 2.0, 8))
        P, I = contract_tables(surf, truth, SUR_GRID)
        p, st = fpe.price_batch(P, I, fpe.BatchOptions(disc=1, precision=0, rtol=1e-9, atol=1e-11,
                                                       complex_solve=2, radau_constants=2))
        assert (st == 0).all()
        surf.prices = p + rng.normal(0.0, noise, p.shape)
        x0 = np.array([1.5, 0.08, 0.45, -0.45, 0.08])
        x_f, i_f = calibrate_fpe(surf, x0, **kw)
        x_s, i_s = calibrate_with_surrogate(surf, pr, x0, max_iter=50, polish="none", quote_noise=noise,
                                            polish_iter=30, fpe_kw=kw)
        x_d, i_d = calibrate_with_surrogate(surf, pr, x0, max_iter=50, polish="defect", fpe_kw=kw)
        x_h, i_h = calibrate_with_surrogate(surf, pr, x0, max_iter=50, polish="hybrid", polish_iter=30, fpe_kw=kw)
        for name, x, inf in (("fpe_only", x_f, i_f), ("surrogate", x_s, i_s), ("defect", x_d, i_d),
                             ("hybrid", x_h, i_h)):
            inf = dict(inf)
            inf["max_rel_param_err"] = float(np.max(np.abs(x - truth) / np.abs(truth)))
            inf["x"] = x.tolist()
            res[name].append(inf)
        surfaces.append(truth.tolist())
    summ = {}
    for name, lst in res.items():
        summ[name] = {"seconds_total": float(sum(d["seconds"] for d in lst)),
                      "fpe_contracts_total": int(sum(d["fpe_contracts"] for d in lst)),
                      "mean_max_rel_param_err": float(np.mean([d["max_rel_param_err"] for d in lst])),
                      "median_max_rel_param_err": float(np.median([d["max_rel_param_err"] for d in lst]))}
    line = {"metric": "Heston calibration wall time: surrogate-in-loop vs FPE-only (same GPU)",
            "value": summ["fpe_only"]["seconds_total"] / summ["defect"]["seconds_total"],
            "unit": "x speed-up", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
            "workload": "calibration",
            "config": {"workload": f"{args.surfaces} seeded surfaces of 15 strikes (K/S0 0.7-1.3) x 8 maturities "
                                   "(0.1-2.0), European calls, FP64 FPE prices + N(0, 1e-4 S0) noise, "
                                   f"{SUR_GRID[0]}x{SUR_GRID[1]} grids; surrogate: LM on the ensemble, one FPE "
                                   "verification, FPE polish only if the FPE residual RMS exceeds 1.5x the noise; "
                                   "defect (the headline): LM on the surrogate corrected by its defect against one FPE "
                                   "pricing of the surface per outer iteration, up to 3; hybrid: FPE residuals with "
                                   "surrogate Jacobians"},
            "summary": summ, "surrogate_only_speedup": summ["fpe_only"]["seconds_total"] / summ["surrogate"]["seconds_total"],
            "hybrid_speedup": summ["fpe_only"]["seconds_total"] / summ["hybrid"]["seconds_total"],
            "truths": surfaces, "runs": res, "surrogate_training": info}
    print(json.dumps(line), flush=True)
    pr.close()
    return 0


def make_barrier_batch(n: int, seed: int):
    """Knock-in contracts on the batched-workload parameter draws: down-and-in
    calls with B/S0 ~ U[0.6, 0.95] and up-and-in puts with B/S0 ~ U[1.05, 1.4]
    (half each), K/S0 ~ U[0.8, 1.2], grids n_s in {48, 64, 96} x n_v in
    {24, 32, 48}; each costs two solves (in-out parity), one of them on the
    domain truncated at B."""
    P, I = make_batch(n, seed)
    rng = np.random.default_rng(seed + 7)
    down = np.arange(n) % 2 == 0
    P[:, 9] = np.where(down, 100.0 * rng.uniform(0.6, 0.95, n), 100.0 * rng.uniform(1.05, 1.4, n))
    I[:, 0] = rng.choice([48, 64, 96], n)
    I[:, 1] = rng.choice([24, 32, 48], n)
    I[:, 2] = np.where(down, 0, 5)
    return P, I


def barrier_measure(fpe, torch, stream, steps: int, warmup: int, precision: int, rtol: float, seed: int,
                    sub_n: int = 32, tight: bool = False) -> dict:
    """The knock-in workload on one GPU: 1024 contracts (2048 solves, grids up
    to 96 x 48, both solves of a pair at the default 0.01 x rtol) in one launch
    sequence, timed with CUDA events on `stream` after `warmup` runs.  Error:
    the mixed-precision prices of a sub_n-contract subsample against the FP64
    path at the same tolerances (the same algorithm as the CPU oracle), and
    with tight=True also against FP64 at rtol 1e-10."""
    nc = 1024
    P, I = make_barrier_batch(nc, seed)
    opts = fpe.BatchOptions(disc=1, precision=precision, rtol=rtol, atol=rtol * 1e-2,
                            complex_solve=2, radau_constants=2)
    arr, keep = fpe.contracts_from_arrays(P, I)
    plan = fpe.Plan(arr, opts, _keep=keep)
    sptr = stream.cuda_stream
    for _ in range(warmup):
        plan.run(sptr)
    torch.cuda.synchronize()
    ktimes = plan.kernel_times(sptr)
    stats = plan.stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_launch = 0
    e0.record(stream)
    for _ in range(steps):
        n_launch += plan.run(sptr)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    p_out, _, _, _, st = plan.results()
    plan.close()
    sub = np.arange(0, nc, nc // sub_n)
    floor = 1e-6 * 100.0
    ref, st_ref = fpe.price_batch(P[sub], I[sub], fpe.BatchOptions(
        disc=1, precision=0, rtol=rtol, atol=rtol * 1e-2, complex_solve=2, radau_constants=2))
    rel = np.abs(p_out[sub] - ref) / np.maximum(np.abs(ref), floor)
    out = {"value": nc / (ms / 1000.0), "unit": "prices/s", "ms_per_step": ms, "steps": steps, "warmup": warmup,
           "contracts": nc, "solves": int(stats["solves"]), "rtol": rtol, "knock_in_tol_scale": 0.01,
           "max_rel_err_vs_fp64_same_tol": float(rel.max()), "subsample": int(len(sub)), "err_floor": floor,
           "status_ok": bool((st == 0).all() and (st_ref == 0).all()), "gpu_launches": n_launch,
           "kernel_ms": {"setup": ktimes[0], "galerkin": ktimes[1], "ic": ktimes[2], "radau": ktimes[3],
                         "payoff": ktimes[4]},
           "solver": {k: int(v) for k, v in stats.items()}}
    if tight:
        tref, _ = fpe.price_batch(P[sub], I[sub], fpe.BatchOptions(
            disc=1, precision=0, rtol=1e-10, atol=1e-12, complex_solve=2, radau_constants=2,
            knock_in_tol_scale=1.0))
        out["max_rel_err_vs_fp64_rtol1e-10"] = float((np.abs(p_out[sub] - tref) / np.maximum(np.abs(tref), floor)).max())
    return out


def run_barrier_workload(args):
    import torch

    import fpe_option_b200 as fpe
    from fpe_option_b200 import build

    build.build_library()
    if not fpe.is_available():
        raise RuntimeError("CUDA engine unavailable")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    with ClockSampler(0) as clk:
        m = barrier_measure(fpe, torch, stream, args.steps, max(args.warmup, 3), args.precision, args.rtol,
                            args.seed, sub_n=64, tight=True)
    line = {"metric": "FPE knock-in prices/sec on 1 B200 (in-out parity, two solves each)",
            "value": m["value"], "unit": "prices/s", "n_gpus": 1, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": m["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "dtype": "f32-factors/f64" if args.precision == 1 else "f64", "data": "synthetic",
            "workload": "barrier",
            "config": {"workload": f"1024 knock-in contracts ({m['solves']} solves), grids 48-96 x 24-48, "
                                   "one launch sequence", **{k: m[k] for k in ("rtol", "knock_in_tol_scale",
                                   "max_rel_err_vs_fp64_same_tol", "max_rel_err_vs_fp64_rtol1e-10", "subsample",
                                   "err_floor", "status_ok")}},
            "gpu_launches": m["gpu_launches"], "kernel_ms": m["kernel_ms"], "solver": m["solver"],
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def C_SIZE_CONTRACT():
    import ctypes

    from fpe_option_b200 import _lib

    return ctypes.sizeof(_lib.FpeContract)


if __name__ == "__main__":
    sys.exit(main())
