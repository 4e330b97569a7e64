// Host side of the B200 Fokker-Planck pricing engine: batch planning, device
// arenas, kernel launches and the C ABI (include/fpe_engine.h).
//
// A contract becomes one device solve, or two for knock-ins (in-out parity,
// reference src/server/pricer.mojo:87-120), plus four bumped pricings when
// Greeks are requested (greeks.mojo:36-53, pricing_engine.mojo:31-39).  All
// solves of a batch run as one CTA each in the same five launches:
//   k_setup -> k_galerkin -> k_ic -> k_radau<FT> -> k_payoff.
// There is no host fallback: without a usable GPU every entry point fails.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/fpe_engine.h"
#include "fpe_device.h"
#include "k_cf.cuh"
#include "k_galerkin.cuh"
#include "k_ic.cuh"
#include "k_interp.cuh"
#include "k_payoff.cuh"
#include "radau_launch.h"
#include "k_setup.cuh"

static_assert(FPE_SOLVE_INFO_WORDS == FPE_INFO_COUNT, "per-solve info words of the C ABI");

// Stage buffers of the staged sweeps (2 .. 4; a solve uses as many as its
// shared scratch holds, up to this).
#ifndef FPE_SWEEP_BUFS
#define FPE_SWEEP_BUFS 2
#endif

// Reads a table of tuned solve shapes (the autotuner's section below).
static void tune_load_file(const char* path);

namespace {

#define CK(x)                                                                       \
  do {                                                                              \
    cudaError_t e_ = (x);                                                           \
    if (e_ != cudaSuccess) {                                                        \
      if (std::getenv("FPE_DEBUG"))                                                 \
        std::fprintf(stderr, "fpe: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(e_), \
                     __FILE__, __LINE__);                                           \
      return -1;                                                                    \
    }                                                                               \
  } while (0)

struct Context {
  bool ok = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  int smem_optin = 0;
};

Context& ctx() {
  static Context c;
  static std::once_flag once;
  std::call_once(once, [] {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return;
    if (cudaGetDevice(&c.device) != cudaSuccess) return;
    if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) return;
    cudaDeviceGetAttribute(&c.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device);
    tune_load_file(std::getenv("FPE_TUNE_TABLE"));
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, c.device) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    int lim = c.smem_optin;
    if (cudaFuncSetAttribute(fpe::k_setup, cudaFuncAttributeMaxDynamicSharedMemorySize, lim) != cudaSuccess) return;
    const int ic_lim = lim - int(sizeof(fpe::IcSmem)) - 1024;
    if (cudaFuncSetAttribute(fpe::k_ic, cudaFuncAttributeMaxDynamicSharedMemorySize, ic_lim) != cudaSuccess) return;
    if (fpe::radau_allow_smem<double>(lim) != cudaSuccess) return;
    if (fpe::radau_allow_smem<float>(lim) != cudaSuccess) return;
    c.ok = true;
  });
  return c;
}

// --------------------------------------------------------------------------
// Contract level (host): validation and parameter revision
// --------------------------------------------------------------------------
struct Pricing {  // one Pricer.price call: contract (possibly bumped)
  double kappa, theta, sigma, rho, r, T, S0, V0, barrier, smin, smax;
  int n_s, n_v, type;
  int strike_begin, n_strikes;  // into the plan's strike list
  bool valid;
  int solve_a = -1, solve_b = -1;  // price = P[a] - P[b] (b = -1: P[a])
};

// option_types.mojo:13-32 + heston_params.mojo:19-33
bool pricing_valid(const Pricing& p, const double* K) {
  // every parameter finite (NaN and Inf fail here, not inside a solve)
  for (double x : {p.kappa, p.theta, p.sigma, p.rho, p.r, p.T, p.S0, p.V0, p.barrier, p.smin, p.smax})
    if (!std::isfinite(x)) return false;
  if (!(p.kappa > 0 && p.theta > 0 && p.sigma > 0 && p.T > 0 && p.S0 > 0 && p.V0 >= 0 &&
        p.smin >= 0 && p.smax > p.smin && p.rho >= -1 && p.rho <= 1))
    return false;
  if (p.type < 0 || p.type > 9 || p.n_strikes <= 0) return false;
  for (int i = 0; i < p.n_strikes; ++i)
    if (!(K[i] > 0.0) || !std::isfinite(K[i])) return false;
  if (p.type <= 3) {
    if (p.barrier <= 0.0 || p.barrier >= p.S0) return false;
  } else if (p.type <= 7) {
    if (p.barrier <= 0.0 || p.barrier < p.S0) return false;
  } else if (p.barrier != 0.0) {
    return false;
  }
  return true;
}

struct Opts {
  int disc = 0, precision = 0, num_insert = 50, refine = 0, ic_sub = 8, greeks = 0;
  int complex_mode = 0;  // resolved: 0 GMRES(10) (reference), 1 direct complex block LU
  int radau_exact = 0;   // resolved: 0 the reference's stage constants, 1 exact Radau IIA
  double rtol = 1e-4, atol = 1e-6, ic_sigma_s = 0.6, ic_sigma_v = 0.004, rel_s = 0.01,
         rel_v = 0.1;
  double max_step = 0.0, first_step = 0.0;  // 0: the reference Pricer's T/5 and 1e-6
  int price_rule = 0;                       // 1: calibration-objective integration
  int max_steps = 0;                        // <= 0: 100000 (radau.mojo:257-263)
  int fp64_retry = 1;                       // re-solve failed mixed solves with FP64 factors
  long long stage_wait = 0;                 // <= 0: about one second
  int block_split = 0;                      // 0 auto, 1 nv x nv blocks, 2 half-width blocks
  double ki_scale = 1.0;                    // tolerance factor of a knock-in's two solves
  int sweep_buffers = 0;                    // 0 auto, 2 .. 4
};

Opts opts_from(const FpeBatchOptions* o, int default_num_insert) {
  Opts r;
  r.num_insert = default_num_insert;
  if (!o) return r;
  r.disc = o->disc;
  r.precision = o->precision;
  if (o->num_insert > 0) r.num_insert = o->num_insert;
  if (o->refine > 0) r.refine = o->refine;
  // complex_solve: 0 auto (GMRES for the reference discretization, direct
  // for the config discretization), 1 GMRES(10), 2 direct complex LU
  r.complex_mode = o->complex_solve == 2 ? 1 : o->complex_solve == 1 ? 0 : (o->disc == 1 ? 1 : 0);
  // radau_constants: 0 auto (reference values on the reference discretization,
  // exact Radau IIA on the config discretization), 1 reference, 2 exact
  r.radau_exact = o->radau_constants == 2 || (o->radau_constants == 0 && o->disc == 1);
  if (o->rtol > 0) r.rtol = o->rtol;
  if (o->atol > 0) r.atol = o->atol;
  if (o->ic_sigma_s > 0) r.ic_sigma_s = o->ic_sigma_s;
  if (o->ic_sigma_v > 0) r.ic_sigma_v = o->ic_sigma_v;
  if (o->ic_sub > 0) r.ic_sub = o->ic_sub;
  r.greeks = o->greeks;
  if (o->rel_s > 0) r.rel_s = o->rel_s;
  if (o->rel_v > 0) r.rel_v = o->rel_v;
  if (o->max_step > 0) r.max_step = o->max_step;
  r.first_step = std::isfinite(o->first_step) ? o->first_step : 0.0;
  r.price_rule = (o->price_rule == 1 && o->disc == 0) ? 1 : 0;
  r.max_steps = o->max_steps > 0 ? o->max_steps : 0;
  r.fp64_retry = o->fp64_retry < 0 ? 0 : 1;
  r.stage_wait = o->stage_wait_cycles > 0 ? (long long)o->stage_wait_cycles : 0;
  r.block_split = (o->block_split == 1 || o->block_split == 2) ? o->block_split : 0;
  r.ki_scale = (o->knock_in_tol_scale > 0.0 && std::isfinite(o->knock_in_tol_scale)) ? o->knock_in_tol_scale
                                                                                    : (o->disc == 1 ? 0.01 : 1.0);
  r.sweep_buffers = (o->sweep_buffers >= 2 && o->sweep_buffers <= 4) ? o->sweep_buffers : 0;
  return r;
}

int grid_count_reference(int num_insert, bool is_v) {  // domain.mojo:20-66 before dedup
  int left = std::max(1, int(num_insert * 0.2));
  int interm = std::max(3, int(num_insert * 0.3));
  int right = std::max(1, int(num_insert * 0.5));
  int i3 = interm / 3;
  int n = left + std::max(1, i3) + std::max(2, i3) + 1 + std::max(1, i3) + right +
          std::max(2, int(num_insert * 0.1));
  if (is_v) n += std::max(2, int(num_insert * 0.2));
  return n;
}

// Build the descriptor of one solve: revised domain (option_types.mojo:34-54),
// boundary conditions (:56-70), capacities.
FpeSolveDesc make_desc(const Pricing& p, int solve_type, double barrier, const Opts& o) {
  FpeSolveDesc d;
  std::memset(&d, 0, sizeof(d));
  d.kappa = p.kappa; d.theta = p.theta; d.sigma = p.sigma; d.rho = p.rho;
  d.r = p.r; d.T = p.T; d.S0 = p.S0; d.V0 = p.V0;
  d.smin = p.smin; d.smax = p.smax;
  if (solve_type <= 3) d.smin = barrier;
  else if (solve_type <= 7) d.smax = barrier;
  d.vmin = 0.0; d.vmax = 1.0;
  d.barrier = barrier;
  d.rtol = o.rtol; d.atol = o.atol;
  d.max_step = o.max_step; d.first_step = o.first_step;
  d.max_steps = o.max_steps;
  d.stage_wait = o.stage_wait;
  d.price_rule = o.price_rule;
  d.ic_sigma_s = o.ic_sigma_s; d.ic_sigma_v = o.ic_sigma_v;
  d.type = solve_type;
  d.n_s = p.n_s; d.n_v = p.n_v;
  const bool up = solve_type >= 4 && solve_type <= 7;
  if (o.disc == 0) {
    d.left_neu = up ? 1 : 0;
    d.right_neu = up ? 0 : 1;
  } else {
    d.left_neu = 0;
    d.right_neu = up ? 0 : 1;
  }
  d.disc = o.disc;
  d.num_insert = o.num_insert;
  d.ic_sub = o.ic_sub;
  d.strike_off = p.strike_begin;
  d.n_strikes = p.n_strikes;
  d.off_traj = -1;
  if (o.disc == 0) {
    d.cap_knot_s = p.n_s + 24;
    d.cap_knot_v = p.n_v + 24;
    d.cap_grid_s = grid_count_reference(o.num_insert, false);
    d.cap_grid_v = grid_count_reference(o.num_insert, true);
    d.cap_q_s = 5 * (d.cap_grid_s - 1);
    d.cap_q_v = 5 * (d.cap_grid_v - 1);
  } else {
    d.cap_knot_s = p.n_s + 6;
    d.cap_knot_v = p.n_v + 6;
    d.cap_grid_s = p.n_s;
    d.cap_grid_v = p.n_v;
    d.cap_q_s = 4 * (p.n_s - 1);
    d.cap_q_v = 4 * (p.n_v - 1);
  }
  d.cap_dof_s = d.cap_knot_s - 6;
  d.cap_dof_v = d.cap_knot_v - 6;
  return d;
}

// The options of a knock-in's two solves (in-out parity, reference
// src/server/pricer.mojo:87-120): the tolerances scaled by ki_scale, since
// the difference of the vanilla and knock-out prices amplifies their
// relative errors by vanilla / knock-in.
Opts knock_in_opts(const Opts& o) {
  Opts r = o;
  r.rtol *= o.ki_scale;
  r.atol *= o.ki_scale;
  return r;
}

}  // namespace

// --------------------------------------------------------------------------
// Plan
// --------------------------------------------------------------------------
struct FpePlan {
  Opts o;
  std::vector<double> strikes;     // per pricing strike lists (host copy)
  std::vector<Pricing> pricings;   // base pricings first, then greeks bumps
  std::vector<int> contract_base;  // contract -> pricing index of the base
  std::vector<int> contract_strike_off, contract_nk;
  std::vector<double> h_s, h_v;    // Greeks bumps per contract
  std::vector<FpeSolveDesc> descs;
  int n_results = 0;
  // device
  FpeSolveDesc* d_descs = nullptr;
  double* d_strikes = nullptr;
  double* d_prices = nullptr;
  int32_t* d_infos = nullptr;
  double* d_arena = nullptr;
  int32_t* d_iarena = nullptr;
  unsigned char* d_farena = nullptr;
  double* d_traj = nullptr;
  int64_t n_d = 0, n_i = 0, n_f = 0, n_traj = 0;
  size_t radau_smem = 0, setup_smem = 0;
  int fac_global = 0;
  size_t ic_smem = 0;
  int n_price_slots = 0;
  // host results
  std::vector<double> h_prices;
  std::vector<int32_t> h_infos;
  bool ran = false, fetched = false;
  bool retry_pending = false;  // results not yet checked for FP64 re-solves
  int n_retried = 0;
  cudaStream_t stream = nullptr;
};

// Dynamic shared memory of one solve in the Radau kernel: the fixed part
// (control block and the 1-D operator factors; *base) plus the real and, for
// the direct complex stage solve, complex factorization scratch of its block
// split (capacities, so the kernel's own decision from the actual sizes never
// asks for more).
static size_t radau_smem_need(const FpeSolveDesc& d, int esz, int cplx, size_t* base) {
  const int nv = std::min(d.cap_dof_v, FPE_MAX_NDOF_V);
  const int ns_cap = std::min(d.cap_dof_s, FPE_MAX_NDOF_S);
  const int m = fpe_blk_split(d.blk_split, nv);
  const size_t el = size_t(fpe_fac_scratch_elems(nv / m, fpe_blk_bw(m)));
  *base = sizeof(fpe::RadauSmem) + size_t(4 * ns_cap * 7 + 5 * nv * 7) * 8 + 64;
  return *base + el * esz + (cplx ? el * 2 * esz + 16 : 0);
}

// --------------------------------------------------------------------------
// Tuned solve shapes.  For a grid class (discretization, n_s, n_v knot
// inputs, factor precision, complex stage mode) the autotuner
// (fpe_option_b200/autotune.py) times the candidate shapes on the device and
// installs the fastest here; a plan's solves look their class up.  The table
// can also be read from a text file named by FPE_TUNE_TABLE at start-up (one
// class per line: disc n_s n_v precision complex_solve block_split
// sweep_buffers).
// --------------------------------------------------------------------------
struct TuneShape {
  int block_split = 0, sweep_buffers = 0;
};
using TuneKey = std::tuple<int, int, int, int, int>;  // disc, n_s, n_v, precision, complex mode

static std::mutex& tune_mu() {
  static std::mutex m;
  return m;
}
static std::map<TuneKey, TuneShape>& tune_table() {
  static std::map<TuneKey, TuneShape> t;
  return t;
}
static bool tune_find(const TuneKey& k, TuneShape* out) {
  std::lock_guard<std::mutex> lock(tune_mu());
  auto it = tune_table().find(k);
  if (it == tune_table().end()) return false;
  *out = it->second;
  return true;
}
static void tune_load_file(const char* path) {
  FILE* f = path ? std::fopen(path, "r") : nullptr;
  if (!f) return;
  char line[256];
  std::lock_guard<std::mutex> lock(tune_mu());
  while (std::fgets(line, sizeof(line), f)) {
    int v[7];
    if (line[0] == '#') continue;
    if (std::sscanf(line, "%d %d %d %d %d %d %d", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5], &v[6]) != 7) continue;
    tune_table()[TuneKey{v[0], v[1], v[2], v[3], v[4]}] = TuneShape{v[5], v[6]};
  }
  std::fclose(f);
}

// The shape of a solve: the caller's explicit choices, else the tuned shape of
// its grid class, else full nv x nv blocks when their factorization scratch
// fits in shared memory and half-width blocks when it does not (nv = 48 in
// mixed precision, for one), with the launch's default stage buffers.
static void resolve_solve_shape(FpeSolveDesc& d, const Opts& o, int esz, size_t optin) {
  TuneShape t;
  const bool tuned = tune_find(TuneKey{o.disc, d.n_s, d.n_v, esz == 8 ? 0 : 1, o.complex_mode}, &t);
  d.sweep_bufs = o.sweep_buffers ? o.sweep_buffers : (tuned ? t.sweep_buffers : 0);
  if (o.block_split) {
    d.blk_split = o.block_split;
    return;
  }
  if (tuned && t.block_split) {
    d.blk_split = t.block_split;
    return;
  }
  d.blk_split = 1;
  size_t base = 0;
  if (radau_smem_need(d, esz, o.complex_mode, &base) > optin) d.blk_split = 2;
}

static int plan_layout(FpePlan* P, int esz) {
  int64_t od = 0, oi = 0, of = 0, ot = 0;
  size_t smem_fit_max = 0, smem_base_max = 0;
  const size_t optin = size_t(ctx().smem_optin > 0 ? ctx().smem_optin : 232448);
  const int cplx = P->o.complex_mode;
  for (auto& d : P->descs) {
    resolve_solve_shape(d, P->o, esz, optin);
    d.off_d = od;
    d.off_i = oi;
    d.off_f = of;
    od += fpe_dlayout(d).total;
    oi += fpe_ilayout(d).total;
    of += fpe_factor_bytes(d, esz, cplx);
    if (d.save_traj) {
      d.off_traj = ot;
      ot += d.traj_cap + int64_t(d.traj_cap) * d.cap_dof_s * d.cap_dof_v;
    }
    size_t base = 0;
    const size_t sm = radau_smem_need(d, esz, cplx, &base);
    smem_base_max = std::max(smem_base_max, base);
    if (sm <= optin) smem_fit_max = std::max(smem_fit_max, sm);
  }
  P->n_d = od;
  P->n_i = oi;
  P->n_f = of;
  P->n_traj = ot;
  // Launch with the largest shared-memory need among the solves whose
  // factorization scratch fits the opt-in limit; each solve that does not fit
  // keeps its scratch in its global work area (decided per solve by the
  // kernel), so one wide grid does not move a whole mixed batch to global.
  P->fac_global = 0;
  P->radau_smem = std::max(smem_fit_max, smem_base_max);
  // ADMM iterates of the IC projection in shared memory, per solve, when they fit
  const size_t ic_lim = optin - sizeof(fpe::IcSmem) - 1024;
  size_t ic = 0;
  for (auto& d : P->descs) {
    const size_t need = fpe_ic_admm_bytes(d.cap_dof_s, d.cap_dof_v);
    if (need <= ic_lim) ic = std::max(ic, need);
  }
  P->ic_smem = ic;
  P->setup_smem = sizeof(fpe::SetupSmem);
  return 0;
}

static int plan_upload(FpePlan* P) {
  Context& C = ctx();
  if (!C.ok) return -1;
  P->stream = C.stream;
  const size_t ns = P->descs.size();
  cudaStream_t s = P->stream;
  CK(cudaMallocAsync(&P->d_descs, std::max<size_t>(ns, 1) * sizeof(FpeSolveDesc), s));
  CK(cudaMallocAsync(&P->d_strikes, std::max<size_t>(P->strikes.size(), 1) * sizeof(double), s));
  CK(cudaMallocAsync(&P->d_prices, std::max<size_t>(P->n_price_slots, 1) * sizeof(double), s));
  CK(cudaMallocAsync(&P->d_infos, std::max<size_t>(ns, 1) * FPE_INFO_COUNT * sizeof(int32_t), s));
  CK(cudaMallocAsync(&P->d_arena, std::max<int64_t>(P->n_d, 1) * sizeof(double), s));
  CK(cudaMallocAsync(&P->d_iarena, std::max<int64_t>(P->n_i, 1) * sizeof(int32_t), s));
  CK(cudaMallocAsync(&P->d_farena, std::max<int64_t>(P->n_f, 256), s));
  if (P->n_traj > 0) CK(cudaMallocAsync(&P->d_traj, P->n_traj * sizeof(double), s));
  if (ns) CK(cudaMemcpyAsync(P->d_descs, P->descs.data(), ns * sizeof(FpeSolveDesc), cudaMemcpyHostToDevice, s));
  if (!P->strikes.empty())
    CK(cudaMemcpyAsync(P->d_strikes, P->strikes.data(), P->strikes.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  return 0;
}

// Stage-wise launch: stages [from, to) of setup(0) galerkin(1) ic(2) radau(3) payoff(4).
static int plan_launch(FpePlan* P, cudaStream_t s, int from, int to) {
  const int ns = int(P->descs.size());
  if (ns == 0) return 0;
  int launches = 0;
  const dim3 grid(ns), block(FPE_BLOCK);
  if (from <= 0 && to > 0) {
    fpe::k_setup<<<grid, block, P->setup_smem, s>>>(P->d_descs, P->d_arena, P->d_iarena, P->d_infos);
    ++launches;
  }
  if (from <= 1 && to > 1) {
    fpe::k_galerkin<<<grid, block, 0, s>>>(P->d_descs, P->d_arena, P->d_iarena, P->d_infos);
    ++launches;
  }
  if (from <= 2 && to > 2) {
    fpe::k_ic<<<grid, block, P->ic_smem, s>>>(P->d_descs, P->d_arena, P->d_iarena, P->d_infos,
                                              P->ic_smem);
    ++launches;
  }
  if (from <= 3 && to > 3) {
    const fpe::RadauConstants rk = fpe::radau_constants(P->o.radau_exact != 0);
    if (P->o.precision == 0) {
      fpe::RadauKernelArgs<double> a{P->d_descs, P->d_arena, P->d_iarena, P->d_infos, P->d_farena,
                                     P->d_traj, 0, P->o.complex_mode, P->fac_global,
                                     rk.u1, rk.alph, rk.beta, rk.ti13, P->radau_smem,
                                     P->o.sweep_buffers ? P->o.sweep_buffers : FPE_SWEEP_BUFS};
      CK(fpe::launch_radau<double>(a, grid, dim3(FPE_RADAU_THREADS), P->radau_smem, s));
    } else {
      fpe::RadauKernelArgs<float> a{P->d_descs, P->d_arena, P->d_iarena, P->d_infos, P->d_farena,
                                    P->d_traj, P->o.refine, P->o.complex_mode, P->fac_global,
                                    rk.u1, rk.alph, rk.beta, rk.ti13, P->radau_smem,
                                     P->o.sweep_buffers ? P->o.sweep_buffers : FPE_SWEEP_BUFS};
      CK(fpe::launch_radau<float>(a, grid, dim3(FPE_RADAU_THREADS), P->radau_smem, s));
    }
    ++launches;
  }
  if (from <= 4 && to > 4) {
    fpe::k_payoff<<<grid, block, 0, s>>>(P->d_descs, P->d_arena, P->d_iarena, P->d_infos, P->d_strikes, P->d_prices);
    ++launches;
  }
  CK(cudaGetLastError());
  return launches;
}

static FpePlan* plan_build(const FpeContract* c, int n, const Opts& o, bool save_traj) {
  auto* P = new FpePlan();
  P->o = o;
  // base pricings
  for (int i = 0; i < n; ++i) {
    const FpeContract& k = c[i];
    Pricing p;
    p.kappa = k.kappa; p.theta = k.theta; p.sigma = k.sigma; p.rho = k.rho;
    p.r = k.r; p.T = k.T; p.S0 = k.S0; p.V0 = k.V0; p.barrier = k.barrier;
    p.smin = k.s_min >= 0.0 ? k.s_min : 0.0;
    p.smax = k.s_max > 0.0 ? k.s_max : k.S0 * 3.0;
    p.n_s = k.n_s; p.n_v = k.n_v; p.type = k.option_type;
    p.strike_begin = int(P->strikes.size());
    p.n_strikes = std::max(0, int(k.n_strikes));
    for (int j = 0; j < p.n_strikes; ++j) P->strikes.push_back(k.strikes[j]);
    p.valid = pricing_valid(p, P->strikes.data() + p.strike_begin) && p.n_s >= 4 && p.n_v >= 4 &&
              p.n_s <= 256 && p.n_v <= 256;
    P->contract_base.push_back(int(P->pricings.size()));
    P->contract_strike_off.push_back(p.strike_begin);
    P->contract_nk.push_back(p.n_strikes);
    P->n_results += p.n_strikes;
    P->pricings.push_back(p);
  }
  if (o.greeks) {  // 4 bumped pricings per contract (greeks.mojo:23-34)
    for (int i = 0; i < n; ++i) {
      const Pricing base = P->pricings[P->contract_base[i]];
      const double hs = o.rel_s * base.S0, hv = o.rel_v * base.V0;
      P->h_s.push_back(hs);
      P->h_v.push_back(hv);
      const double bs[4] = {hs, -hs, 0.0, 0.0}, bv[4] = {0.0, 0.0, hv, -hv};
      for (int b = 0; b < 4; ++b) {
        Pricing p = base;
        p.S0 = base.S0 + bs[b];
        p.V0 = base.V0 + bv[b];
        p.valid = pricing_valid(p, P->strikes.data() + p.strike_begin) && base.valid;
        P->pricings.push_back(p);
      }
    }
  }
  // solves
  for (auto& p : P->pricings) {
    if (p.valid && grid_count_reference(o.num_insert, true) > 8192 && o.disc == 0) p.valid = false;
    if (!p.valid) continue;
    const int ot = p.type;
    if (ot == 0 || ot == 1 || ot == 4 || ot == 5) {
      const bool call = ot % 2 == 0, down = ot <= 1;
      int out_type = (down ? 2 : 6) + (call ? 0 : 1);
      const Opts oki = knock_in_opts(o);
      p.solve_a = int(P->descs.size());
      P->descs.push_back(make_desc(p, call ? 8 : 9, 0.0, oki));
      p.solve_b = int(P->descs.size());
      P->descs.push_back(make_desc(p, out_type, p.barrier, oki));
    } else {
      p.solve_a = int(P->descs.size());
      P->descs.push_back(make_desc(p, ot, p.barrier, o));
    }
  }
  // Launch the solves longest first.  One CTA runs one solve to completion and
  // the block scheduler hands out CTAs in index order, so ordering by the
  // estimated cost (stage factorization ~ ns nv^3, step count growing slowly
  // with T) is longest-processing-time list scheduling over the SMs.
  if (P->descs.size() > 1) {
    const size_t n = P->descs.size();
    std::vector<double> cost(n);
    for (size_t s = 0; s < n; ++s) {
      const FpeSolveDesc& d = P->descs[s];
      const double ns = d.cap_dof_s, nv = d.cap_dof_v;
      cost[s] = ns * nv * nv * (nv + 8.0) * (1.0 + 0.2 * std::log1p(d.T / 0.1));
    }
    std::vector<int> perm(n), pos(n);
    for (size_t s = 0; s < n; ++s) perm[s] = int(s);
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<FpeSolveDesc> sorted(n);
    for (size_t k = 0; k < n; ++k) {
      sorted[k] = P->descs[perm[k]];
      pos[perm[k]] = int(k);
    }
    P->descs.swap(sorted);
    for (auto& p : P->pricings) {
      if (p.solve_a >= 0) p.solve_a = pos[p.solve_a];
      if (p.solve_b >= 0) p.solve_b = pos[p.solve_b];
    }
  }
  // each solve prices into its own slot range
  int slot = 0;
  for (auto& d : P->descs) {
    d.strike_off = d.strike_off;  // strikes read from the pricing's list
    d.save_traj = save_traj ? 1 : 0;
    d.traj_cap = save_traj ? 2048 : 0;
    slot += d.n_strikes;
  }
  P->n_price_slots = slot;
  plan_layout(P, o.precision == 0 ? 8 : 4);
  return P;
}

// price slot of solve s, strike j: solves are laid out in descriptor order.
static void price_slots(const FpePlan* P, std::vector<int>& first) {
  first.resize(P->descs.size());
  int slot = 0;
  for (size_t s = 0; s < P->descs.size(); ++s) {
    first[s] = slot;
    slot += P->descs[s].n_strikes;
  }
}

static int plan_prepare_prices(FpePlan* P) {
  // k_payoff writes prices[d.strike_off + k]; remap each solve to its own slots.
  std::vector<int> first;
  price_slots(P, first);
  for (size_t s = 0; s < P->descs.size(); ++s) P->descs[s].strike_off = first[s];
  // strikes array laid out per solve as well
  std::vector<double> per_solve(P->n_price_slots);
  for (auto& p : P->pricings) {
    for (int sidx : {p.solve_a, p.solve_b}) {
      if (sidx < 0) continue;
      for (int j = 0; j < p.n_strikes; ++j) per_solve[first[sidx] + j] = P->strikes[p.strike_begin + j];
    }
  }
  P->strikes.swap(per_solve);
  // keep the original per-pricing strike offsets valid for result combination
  return 0;
}

static int plan_fetch(FpePlan* P) {
  if (P->fetched) return 0;
  const size_t ns = P->descs.size();
  P->h_prices.assign(P->n_price_slots, 0.0);
  P->h_infos.assign(ns * FPE_INFO_COUNT, 0);
  if (ns) {
    CK(cudaMemcpyAsync(P->h_prices.data(), P->d_prices, P->n_price_slots * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
    CK(cudaMemcpyAsync(P->h_infos.data(), P->d_infos, ns * FPE_INFO_COUNT * sizeof(int32_t), cudaMemcpyDeviceToHost, P->stream));
  }
  CK(cudaStreamSynchronize(P->stream));
  P->fetched = true;
  return 0;
}

static void plan_free(FpePlan* P) {
  if (!P) return;
  cudaStream_t s = P->stream;
  void* ptrs[] = {P->d_descs, P->d_strikes, P->d_prices, P->d_infos, P->d_arena, P->d_iarena, P->d_farena, P->d_traj};
  for (void* p : ptrs)
    if (p) cudaFreeAsync(p, s);
  if (s) cudaStreamSynchronize(s);
  delete P;
}

// Combine solve prices into per-strike pricing values (parity) and Greeks.
static int plan_combine(FpePlan* P, double* prices, double* delta, double* gamma, double* vega,
                        int32_t* status) {
  std::vector<int> first;
  price_slots(P, first);
  int worst = 0;
  auto pricing_values = [&](const Pricing& p, std::vector<double>& out, std::vector<int>& st) {
    out.assign(p.n_strikes, 0.0);
    st.assign(p.n_strikes, p.valid ? 0 : FPE_STATUS_INVALID);
    if (!p.valid) return;
    for (int j = 0; j < p.n_strikes; ++j) {
      double v = P->h_prices[first[p.solve_a] + j];
      int sa = P->h_infos[size_t(p.solve_a) * FPE_INFO_COUNT + FPE_INFO_STATUS];
      int sb = 0;
      if (p.solve_b >= 0) {
        v -= P->h_prices[first[p.solve_b] + j];
        sb = P->h_infos[size_t(p.solve_b) * FPE_INFO_COUNT + FPE_INFO_STATUS];
      }
      out[j] = v;
      st[j] = sa ? sa : sb;
    }
  };
  const int nc = int(P->contract_base.size());
  int r = 0;
  std::vector<double> base, up, dn, upv, dnv;
  std::vector<int> st, st2;
  for (int c = 0; c < nc; ++c) {
    const Pricing& p = P->pricings[P->contract_base[c]];
    pricing_values(p, base, st);
    for (int j = 0; j < p.n_strikes; ++j) {
      if (prices) prices[r + j] = base[j];
      if (status) status[r + j] = st[j];
      if (st[j] && !worst) worst = st[j];
    }
    if (P->o.greeks) {
      const int g0 = nc + 4 * c;
      pricing_values(P->pricings[g0 + 0], up, st2);
      pricing_values(P->pricings[g0 + 1], dn, st2);
      pricing_values(P->pricings[g0 + 2], upv, st2);
      pricing_values(P->pricings[g0 + 3], dnv, st2);
      const double hs = P->h_s[c], hv = P->h_v[c];
      const double i2h = 1.0 / (2.0 * hs), ih2 = 1.0 / (hs * hs), i2v = 1.0 / (2.0 * hv);
      for (int j = 0; j < p.n_strikes; ++j) {  // simd_utils.mojo:23-60
        if (delta) delta[r + j] = p.valid ? (up[j] - dn[j]) * i2h : 0.0;
        if (gamma) gamma[r + j] = p.valid ? (up[j] - 2.0 * base[j] + dn[j]) * ih2 : 0.0;
        if (vega) vega[r + j] = p.valid ? (upv[j] - dnv[j]) * i2v : 0.0;
      }
    }
    r += p.n_strikes;
  }
  return worst;
}

// A mixed-precision solve that ends with a solver failure (a singular or
// non-finite FP32 factor, the step caps, a sweep's wait that gave up) is
// solved again with FP64 factors: the failed solves' descriptors form one
// sub-plan that runs all five phases, and its prices and status words replace
// the first attempt's.  Returns the number of re-solved solves, < 0 on error.
static bool solver_failure(int st) { return st >= FPE_ERR_SINGULAR && st <= FPE_ERR_TIMEOUT; }

static int plan_retry_fp64(FpePlan* P) {
  if (P->o.precision == 0 || !P->o.fp64_retry) return 0;
  std::vector<int> first, fail;
  price_slots(P, first);
  for (size_t s = 0; s < P->descs.size(); ++s)
    if (solver_failure(P->h_infos[s * FPE_INFO_COUNT + FPE_INFO_STATUS])) fail.push_back(int(s));
  if (fail.empty()) return 0;
  auto* R = new FpePlan();
  R->o = P->o;
  R->o.precision = 0;
  int slot = 0;
  for (int s : fail) {
    FpeSolveDesc d = P->descs[s];
    d.stage_wait = 0;  // the default bounded wait
    d.strike_off = slot;
    for (int j = 0; j < d.n_strikes; ++j) R->strikes.push_back(P->strikes[first[s] + j]);
    slot += d.n_strikes;
    R->descs.push_back(d);
  }
  R->n_price_slots = slot;
  plan_layout(R, 8);
  int rc = plan_upload(R);
  if (rc == 0 && plan_launch(R, R->stream, 0, 5) < 0) rc = -1;
  if (rc == 0 && plan_fetch(R) < 0) rc = -1;
  if (rc == 0) {
    for (size_t k = 0; k < fail.size(); ++k) {
      const int s = fail[k];
      for (int j = 0; j < P->descs[s].n_strikes; ++j)
        P->h_prices[first[s] + j] = R->h_prices[R->descs[k].strike_off + j];
      std::memcpy(&P->h_infos[size_t(s) * FPE_INFO_COUNT], &R->h_infos[k * FPE_INFO_COUNT],
                  FPE_INFO_COUNT * sizeof(int32_t));
    }
  }
  plan_free(R);
  return rc < 0 ? -1 : int(fail.size());
}

// --------------------------------------------------------------------------
// Stepwise pipeline (reference src/server/compute_pipeline.mojo:17-171)
// --------------------------------------------------------------------------
struct FpeCompute {
  FpeContract c;
  double S0_strike;
  Opts o;
  Pricing revised;  // fp.revised_heston() parameters
  FpePlan* plan = nullptr;  // the pipeline's own solve (revised domain)
  int stage = 0;            // stages completed
  double* d_pdf = nullptr;
};

static int compute_run(FpeCompute* h, int upto) {
  FpePlan* P = h->plan;
  if (h->stage >= upto) return 0;
  if (plan_launch(P, P->stream, h->stage, upto) < 0) return -1;
  CK(cudaStreamSynchronize(P->stream));
  h->stage = upto;
  P->fetched = false;
  if (plan_fetch(P) < 0) return -1;
  int st = P->h_infos[FPE_INFO_STATUS];
  return (st == 0 || st == FPE_ERR_MAX_STEPS || st == FPE_ERR_STEP_UNDERFLOW) ? 0 : -1;
}

template <typename T>
static T* dup_host(const std::vector<T>& v) {
  if (v.empty()) return nullptr;
  T* p = static_cast<T*>(std::malloc(v.size() * sizeof(T)));
  std::memcpy(p, v.data(), v.size() * sizeof(T));
  return p;
}

static int fetch_doubles(FpeCompute* h, int64_t off, int64_t n, std::vector<double>& out) {
  out.resize(n);
  if (n == 0) return 0;
  CK(cudaMemcpy(out.data(), h->plan->d_arena + h->plan->descs[0].off_d + off, n * sizeof(double),
                cudaMemcpyDeviceToHost));
  return 0;
}

static int info_of(FpeCompute* h, int k) { return h->plan->h_infos[k]; }

static FpeCompute* compute_create(const FpeContract& k, const Opts& o) {
  if (!ctx().ok) return nullptr;
  Pricing p;
  p.kappa = k.kappa; p.theta = k.theta; p.sigma = k.sigma; p.rho = k.rho;
  p.r = k.r; p.T = k.T; p.S0 = k.S0; p.V0 = k.V0; p.barrier = k.barrier;
  p.smin = k.s_min >= 0.0 ? k.s_min : 0.0;
  p.smax = k.s_max > 0.0 ? k.s_max : k.S0 * 3.0;
  p.n_s = k.n_s; p.n_v = k.n_v; p.type = k.option_type;
  p.strike_begin = 0;
  p.n_strikes = 1;
  double s0 = k.S0;
  p.valid = pricing_valid(p, &s0) && p.n_s >= 4 && p.n_v >= 4 && p.n_s <= 256 && p.n_v <= 256;
  // the setup kernel sorts each raw reference grid in an 8192-entry shared buffer
  if (o.disc == 0 && grid_count_reference(o.num_insert, true) > 8192) p.valid = false;
  if (!p.valid) return nullptr;
  auto* h = new FpeCompute();
  h->c = k;
  h->S0_strike = k.S0;
  h->c.strikes = &h->S0_strike;
  h->c.n_strikes = 1;
  h->o = o;
  // revised parameters: the pipeline solves on the barrier-truncated domain
  h->revised = p;
  if (p.type <= 3) h->revised.smin = p.barrier;
  else if (p.type <= 7) h->revised.smax = p.barrier;
  auto* P = new FpePlan();
  P->o = o;
  P->strikes = {k.S0};
  P->pricings.push_back(p);
  FpeSolveDesc d = make_desc(p, p.type, p.barrier, o);
  d.save_traj = 1;
  d.traj_cap = 2048;
  P->descs.push_back(d);
  P->n_price_slots = 1;
  plan_layout(P, o.precision == 0 ? 8 : 4);
  P->descs[0].strike_off = 0;
  if (plan_upload(P) < 0) {
    plan_free(P);
    delete h;
    return nullptr;
  }
  h->plan = P;
  if (compute_run(h, 2) < 0) {  // domain, basis, M and K eagerly (compute_pipeline.mojo:29-48)
    plan_free(P);
    delete h;
    return nullptr;
  }
  return h;
}

// Price strikes through a fresh batch (used for knock-ins and Greeks bumps,
// compute_pipeline.mojo:116-128 / greeks.mojo:36-53).
static int price_fresh(const FpeContract& k, const Opts& o, const double* K, int nK, double* out,
                       double* d, double* g, double* v) {
  FpeContract c = k;
  c.strikes = K;
  c.n_strikes = nK;
  Opts oo = o;
  oo.greeks = (d || g || v) ? 1 : 0;
  FpePlan* P = plan_build(&c, 1, oo, false);
  plan_prepare_prices(P);
  int rc = plan_upload(P);
  if (rc == 0 && plan_launch(P, P->stream, 0, 5) < 0) rc = -1;
  if (rc == 0 && plan_fetch(P) < 0) rc = -1;
  if (rc == 0 && plan_retry_fp64(P) < 0) rc = -1;
  std::vector<int32_t> st(nK);
  if (rc == 0) plan_combine(P, out, d, g, v, st.data());
  plan_free(P);
  return rc;
}

static int compute_price(FpeCompute* h, const double* K, int nK, double* out) {
  const int ot = h->c.option_type;
  Opts o = h->o;
  o.rtol = 1e-4;
  o.atol = 1e-6;
  if (ot == 0 || ot == 1 || ot == 4 || ot == 5) return price_fresh(h->c, o, K, nK, out, nullptr, nullptr, nullptr);
  if (compute_run(h, 4) < 0) return -1;
  FpePlan* P = h->plan;
  // re-point the payoff at the requested strikes
  double* d_k = nullptr;
  double* d_p = nullptr;
  cudaStream_t s = P->stream;
  CK(cudaMallocAsync(&d_k, std::max(nK, 1) * sizeof(double), s));
  CK(cudaMallocAsync(&d_p, std::max(nK, 1) * sizeof(double), s));
  CK(cudaMemcpyAsync(d_k, K, nK * sizeof(double), cudaMemcpyHostToDevice, s));
  FpeSolveDesc d = P->descs[0];
  d.strike_off = 0;
  d.n_strikes = nK;
  FpeSolveDesc* d_desc = nullptr;
  CK(cudaMallocAsync(&d_desc, sizeof(d), s));
  CK(cudaMemcpyAsync(d_desc, &d, sizeof(d), cudaMemcpyHostToDevice, s));
  fpe::k_payoff<<<1, FPE_BLOCK, 0, s>>>(d_desc, P->d_arena, P->d_iarena, P->d_infos, d_k, d_p);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, d_p, nK * sizeof(double), cudaMemcpyDeviceToHost, s));
  cudaFreeAsync(d_k, s);
  cudaFreeAsync(d_p, s);
  cudaFreeAsync(d_desc, s);
  CK(cudaStreamSynchronize(s));
  return 0;
}

// ==========================================================================
// C ABI
// ==========================================================================
extern "C" {

int32_t fpe_device_available(void) { return ctx().ok ? 1 : 0; }

FpePlan* fpe_plan_create(const FpeContract* contracts, int32_t n, const FpeBatchOptions* opt) {
  if (!ctx().ok || n < 0 || (n > 0 && !contracts)) return nullptr;
  for (int i = 0; i < n; ++i)
    if (contracts[i].n_strikes < 0 || contracts[i].n_strikes > FPE_MAX_STRIKES ||
        (contracts[i].n_strikes > 0 && !contracts[i].strikes))
      return nullptr;
  FpePlan* P = plan_build(contracts, n, opts_from(opt, 50), false);
  plan_prepare_prices(P);
  if (plan_upload(P) < 0) {
    plan_free(P);
    return nullptr;
  }
  return P;
}

int32_t fpe_plan_run(FpePlan* P, void* stream) {
  if (!P) return -1;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : P->stream;
  if (s != P->stream) {
    // order the plan's uploads before work on the caller's stream
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CK(cudaEventRecord(ev, P->stream));
    CK(cudaStreamWaitEvent(s, ev, 0));
    cudaEventDestroy(ev);
  }
  P->fetched = false;
  P->retry_pending = true;
  int n = plan_launch(P, s, 0, 5);
  if (n < 0) return -1;
  if (s != P->stream) {
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CK(cudaEventRecord(ev, s));
    CK(cudaStreamWaitEvent(P->stream, ev, 0));
    cudaEventDestroy(ev);
  }
  P->ran = true;
  return n;
}

int32_t fpe_plan_results(FpePlan* P, double* prices, double* delta, double* gamma, double* vega,
                         int32_t* status) {
  if (!P || !P->ran) return -1;
  if (plan_fetch(P) < 0) return -1;
  if (P->retry_pending) {
    P->retry_pending = false;
    P->n_retried = plan_retry_fp64(P);
    if (P->n_retried < 0) return -1;
  }
  return plan_combine(P, prices, delta, gamma, vega, status);
}

int32_t fpe_plan_retried(FpePlan* P) { return P ? P->n_retried : -1; }

int32_t fpe_tune_set(int32_t disc, int32_t n_s, int32_t n_v, int32_t precision, int32_t complex_solve,
                     int32_t block_split, int32_t sweep_buffers) {
  if (block_split < 0 || block_split > 2 || (sweep_buffers != 0 && (sweep_buffers < 2 || sweep_buffers > 4)))
    return -1;
  const int cm = complex_solve == 2 ? 1 : complex_solve == 1 ? 0 : (disc == 1 ? 1 : 0);
  std::lock_guard<std::mutex> lock(tune_mu());
  tune_table()[TuneKey{disc, n_s, n_v, precision ? 1 : 0, cm}] = TuneShape{block_split, sweep_buffers};
  return 0;
}

int32_t fpe_tune_get(int32_t disc, int32_t n_s, int32_t n_v, int32_t precision, int32_t complex_solve,
                     int32_t* block_split, int32_t* sweep_buffers) {
  const int cm = complex_solve == 2 ? 1 : complex_solve == 1 ? 0 : (disc == 1 ? 1 : 0);
  TuneShape t;
  if (!tune_find(TuneKey{disc, n_s, n_v, precision ? 1 : 0, cm}, &t)) return 0;
  if (block_split) *block_split = t.block_split;
  if (sweep_buffers) *sweep_buffers = t.sweep_buffers;
  return 1;
}

void fpe_tune_clear(void) {
  std::lock_guard<std::mutex> lock(tune_mu());
  tune_table().clear();
}

int32_t fpe_plan_solve_info(FpePlan* P, int32_t* out) {
  if (!P || !out) return -1;
  if (plan_fetch(P) < 0) return -1;
  std::memcpy(out, P->h_infos.data(), P->h_infos.size() * sizeof(int32_t));
  return int32_t(P->descs.size());
}

int32_t fpe_plan_stats(FpePlan* P, int64_t* out) {
  if (!P || !out) return -1;
  if (plan_fetch(P) < 0) return -1;
  for (int k = 0; k < 20; ++k) out[k] = 0;
  out[0] = int64_t(P->descs.size());
  for (size_t s = 0; s < P->descs.size(); ++s) {
    const int32_t* in = &P->h_infos[s * FPE_INFO_COUNT];
    out[1] += in[FPE_INFO_ACCEPTED];
    out[2] += in[FPE_INFO_REJECTED];
    out[3] += in[FPE_INFO_NEWTON];
    out[4] += in[FPE_INFO_GMRES];
    out[5] += in[FPE_INFO_LU];
    out[6] += in[FPE_INFO_ADMM];
    out[7] = std::max<int64_t>(out[7], in[FPE_INFO_NDOF_S]);
    out[8] = std::max<int64_t>(out[8], in[FPE_INFO_NDOF_V]);
    out[9] += int64_t(in[FPE_INFO_NDOF_S]) * in[FPE_INFO_NDOF_V];
    // algorithmic stage-factor bytes: each LU writes R (+ C) once, each sweep
    // reads the whole real (R) or complex (C = 2R) factor once
    const int64_t nv = in[FPE_INFO_NDOF_V], ns = in[FPE_INFO_NDOF_S];
    const int64_t R = ns * 7 * nv * nv * (P->o.precision == 0 ? 8 : 4);
    const int64_t Cb = P->o.complex_mode ? 2 * R : 0;
    out[10] += in[FPE_INFO_PASS_REAL];
    out[11] += in[FPE_INFO_PASS_CPLX];
    out[12] += int64_t(in[FPE_INFO_PASS_REAL]) * R + int64_t(in[FPE_INFO_PASS_CPLX]) * Cb +
               int64_t(in[FPE_INFO_LU]) * (R + Cb);
    out[13] = std::max<int64_t>(out[13], in[FPE_INFO_STATUS]);
    out[14] += in[FPE_INFO_T_FACTOR];
    out[15] += in[FPE_INFO_T_SOLVE];
    out[16] += in[FPE_INFO_T_KRON];
    out[17] += in[FPE_INFO_T_TOTAL];
    out[18] += in[FPE_INFO_T_FGJ];
    out[19] += in[FPE_INFO_T_FGEMM];
  }
  return 0;
}

int32_t fpe_plan_kernel_times(FpePlan* P, void* stream, float* ms) {
  if (!P || !ms) return -1;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : P->stream;
  cudaEvent_t ev[6];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  if (s != P->stream) {
    CK(cudaEventRecord(ev[0], P->stream));
    CK(cudaStreamWaitEvent(s, ev[0], 0));
  }
  P->fetched = false;
  P->retry_pending = true;
  for (int k = 0; k < 5; ++k) {
    CK(cudaEventRecord(ev[k], s));
    if (plan_launch(P, s, k, k + 1) < 0) return -1;
  }
  CK(cudaEventRecord(ev[5], s));
  CK(cudaEventSynchronize(ev[5]));
  for (int k = 0; k < 5; ++k) CK(cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]));
  for (auto& e : ev) cudaEventDestroy(e);
  P->ran = true;
  return 5;
}

int32_t fpe_plan_sizes(FpePlan* P, int32_t* n_results, int32_t* n_solves) {
  if (!P) return -1;
  if (n_results) *n_results = P->n_results;
  if (n_solves) *n_solves = int32_t(P->descs.size());
  return 0;
}

void fpe_plan_destroy(FpePlan* P) { plan_free(P); }

int32_t fpe_price_batch(const FpeContract* contracts, int32_t n, const FpeBatchOptions* opt,
                        double* prices, double* delta, double* gamma, double* vega, int32_t* status) {
  FpePlan* P = fpe_plan_create(contracts, n, opt);
  if (!P) return -1;
  int rc = fpe_plan_run(P, nullptr) < 0 ? -1 : fpe_plan_results(P, prices, delta, gamma, vega, status);
  plan_free(P);
  return rc;
}

FpeCompute* fpe_compute_create_ex(double kappa, double theta, double sigma, double rho, double r,
                                  double T, double S0, double V0, int32_t n_s, int32_t n_v,
                                  double barrier, int32_t option_type, double s_min, double s_max,
                                  const FpeBatchOptions* opt) {
  FpeContract k{kappa, theta, sigma, rho, r, T, S0, V0, barrier, s_min, s_max, n_s, n_v, option_type, 0, nullptr};
  Opts o = opts_from(opt, 251);
  if (!opt || opt->rtol <= 0) o.rtol = 1e-4;
  if (!opt || opt->atol <= 0) o.atol = 1e-6;
  return compute_create(k, o);
}

FpeCompute* fpe_compute_create(double kappa, double theta, double sigma, double rho, double r,
                               double T, double S0, double V0, int32_t n_s, int32_t n_v,
                               double barrier, int32_t option_type, int32_t num_insert,
                               double s_min, double s_max) {
  FpeBatchOptions o;
  std::memset(&o, 0, sizeof(o));
  o.num_insert = num_insert > 0 ? num_insert : 251;
  return fpe_compute_create_ex(kappa, theta, sigma, rho, r, T, S0, V0, n_s, n_v, barrier,
                               option_type, s_min, s_max, &o);
}

void fpe_compute_destroy(FpeCompute* h) {
  if (!h) return;
  if (h->d_pdf) cudaFree(h->d_pdf);
  plan_free(h->plan);
  delete h;
}

void fpe_compute_knots(FpeCompute* h, FpeVec2Result* res) {
  *res = FpeVec2Result{nullptr, 0, nullptr, 0};
  if (!h) return;
  const FpeDLayout L = fpe_dlayout(h->plan->descs[0]);
  std::vector<double> s, v;
  if (fetch_doubles(h, L.knot_s, info_of(h, FPE_INFO_NKNOT_S), s) < 0) return;
  if (fetch_doubles(h, L.knot_v, info_of(h, FPE_INFO_NKNOT_V), v) < 0) return;
  *res = FpeVec2Result{dup_host(s), int32_t(s.size()), dup_host(v), int32_t(v.size())};
}

void fpe_compute_grid_points(FpeCompute* h, FpeGridPtsResult* res) {
  *res = FpeGridPtsResult{nullptr, 0, nullptr, 0, nullptr, nullptr};
  if (!h) return;
  const FpeDLayout L = fpe_dlayout(h->plan->descs[0]);
  const int nqs = info_of(h, FPE_INFO_NQ_S), nqv = info_of(h, FPE_INFO_NQ_V);
  std::vector<double> s, v, sw, vw;
  if (fetch_doubles(h, L.qp_s, nqs, s) < 0 || fetch_doubles(h, L.qp_v, nqv, v) < 0 ||
      fetch_doubles(h, L.qw_s, nqs, sw) < 0 || fetch_doubles(h, L.qw_v, nqv, vw) < 0)
    return;
  *res = FpeGridPtsResult{dup_host(s), nqs, dup_host(v), nqv, dup_host(sw), dup_host(vw)};
}

void fpe_compute_initial_condition(FpeCompute* h, FpeVecResult* res) {
  *res = FpeVecResult{nullptr, 0};
  if (!h || compute_run(h, 3) < 0) return;
  const FpeDLayout L = fpe_dlayout(h->plan->descs[0]);
  const int N = info_of(h, FPE_INFO_NDOF_S) * info_of(h, FPE_INFO_NDOF_V);
  std::vector<double> q;
  if (fetch_doubles(h, L.q0, N, q) < 0) return;
  *res = FpeVecResult{dup_host(q), int32_t(q.size())};
}

void fpe_compute_solve(FpeCompute* h, FpeMatResult* res) {
  *res = FpeMatResult{nullptr, 0, 0};
  if (!h || compute_run(h, 4) < 0) return;
  FpePlan* P = h->plan;
  const int N = info_of(h, FPE_INFO_NDOF_S) * info_of(h, FPE_INFO_NDOF_V);
  const int ns = info_of(h, FPE_INFO_NSAVED);
  const FpeSolveDesc& d = P->descs[0];
  std::vector<double> all(size_t(ns) * N);
  if (ns > 0 && cudaMemcpy(all.data(), P->d_traj + d.off_traj + d.traj_cap, all.size() * sizeof(double),
                           cudaMemcpyDeviceToHost) != cudaSuccess)
    return;
  *res = FpeMatResult{dup_host(all), ns, N};
}

void fpe_compute_pdf(FpeCompute* h, FpeMatResult* res) {
  *res = FpeMatResult{nullptr, 0, 0};
  if (!h || compute_run(h, 4) < 0) return;
  FpePlan* P = h->plan;
  const int nqs = info_of(h, FPE_INFO_NQ_S), nqv = info_of(h, FPE_INFO_NQ_V);
  const size_t n = size_t(nqs) * nqv;
  if (!h->d_pdf && cudaMalloc(&h->d_pdf, std::max<size_t>(n, 1) * sizeof(double)) != cudaSuccess) return;
  fpe::k_pdf<<<296, 256, 0, P->stream>>>(P->d_descs, P->d_arena, P->d_iarena, P->d_infos, 0, h->d_pdf);
  if (cudaGetLastError() != cudaSuccess) return;
  std::vector<double> out(n);
  if (cudaMemcpyAsync(out.data(), h->d_pdf, n * sizeof(double), cudaMemcpyDeviceToHost, P->stream) != cudaSuccess) return;
  if (cudaStreamSynchronize(P->stream) != cudaSuccess) return;
  *res = FpeMatResult{dup_host(out), nqs, nqv};
}

void fpe_compute_price(FpeCompute* h, const double* K, int32_t n_K, FpeVecResult* res) {
  *res = FpeVecResult{nullptr, 0};
  if (!h || n_K < 0) return;
  std::vector<double> out(n_K);
  if (n_K > 0 && compute_price(h, K, n_K, out.data()) < 0) return;
  *res = FpeVecResult{dup_host(out), n_K};
}

void fpe_compute_greeks(FpeCompute* h, const double* K, int32_t n_K, double rel_s, double rel_v,
                        FpeGreeksResult* res) {
  *res = FpeGreeksResult{nullptr, nullptr, nullptr, 0};
  if (!h || n_K < 0) return;
  // compute_pipeline.mojo:153-171: base from price_at, bumps on the revised parameters
  std::vector<double> base(n_K), d(n_K), g(n_K), v(n_K), tmp(n_K);
  if (n_K > 0 && compute_price(h, K, n_K, base.data()) < 0) return;
  Opts o = h->o;
  o.rtol = 1e-4;
  o.atol = 1e-6;
  o.rel_s = rel_s != 0.0 ? rel_s : 0.01;
  o.rel_v = rel_v != 0.0 ? rel_v : 0.1;
  FpeContract k = h->c;
  k.s_min = h->revised.smin;
  k.s_max = h->revised.smax;
  const double hs = o.rel_s * k.S0, hv = o.rel_v * k.V0;
  std::vector<double> up(n_K), dn(n_K), upv(n_K), dnv(n_K);
  struct B { double ds, dv; std::vector<double>* out; } bumps[4] = {
      {hs, 0, &up}, {-hs, 0, &dn}, {0, hv, &upv}, {0, -hv, &dnv}};
  for (auto& b : bumps) {
    FpeContract kb = k;
    kb.S0 = k.S0 + b.ds;
    kb.V0 = k.V0 + b.dv;
    if (n_K > 0 && price_fresh(kb, o, K, n_K, b.out->data(), nullptr, nullptr, nullptr) < 0) return;
  }
  for (int j = 0; j < n_K; ++j) {
    d[j] = (up[j] - dn[j]) * (1.0 / (2.0 * hs));
    g[j] = (up[j] - 2.0 * base[j] + dn[j]) * (1.0 / (hs * hs));
    v[j] = (upv[j] - dnv[j]) * (1.0 / (2.0 * hv));
  }
  *res = FpeGreeksResult{dup_host(d), dup_host(g), dup_host(v), n_K};
}

void fpe_price_oneshot(double kappa, double theta, double sigma, double rho, double r, double T,
                       double S0, double V0, const double* K, int32_t n_K, double barrier,
                       int32_t option_type, int32_t n_s, int32_t n_v, int32_t num_insert,
                       double s_min, double s_max, FpeOneshotResult* res) {
  *res = FpeOneshotResult{nullptr, nullptr, nullptr, nullptr, 0};
  if (n_K < 0 || !ctx().ok) return;
  FpeContract k{kappa, theta, sigma, rho, r, T, S0, V0, barrier, s_min, s_max, n_s, n_v, option_type, n_K, K};
  FpeBatchOptions o;
  std::memset(&o, 0, sizeof(o));
  o.num_insert = num_insert > 0 ? num_insert : 50;
  o.greeks = 1;
  std::vector<double> p(n_K), d(n_K), g(n_K), v(n_K);
  std::vector<int32_t> st(n_K);
  int rc = fpe_price_batch(&k, 1, &o, p.data(), d.data(), g.data(), v.data(), st.data());
  if (rc < 0) return;
  *res = FpeOneshotResult{dup_host(p), dup_host(d), dup_host(g), dup_host(v), n_K};
}

int64_t fpe_compute_basis_csr(FpeCompute* h, int32_t which, int32_t* n_rows, int32_t* n_cols,
                              int32_t* indptr, int32_t* indices, double* data) {
  if (!h) return -1;
  FpePlan* P = h->plan;
  const FpeSolveDesc& d = P->descs[0];
  const FpeDLayout L = fpe_dlayout(d);
  const FpeILayout IL = fpe_ilayout(d);
  const bool is_v = which >= 2;
  const bool deriv = which == 1 || which == 3;
  const int nq = info_of(h, is_v ? FPE_INFO_NQ_V : FPE_INFO_NQ_S);
  const int nd = info_of(h, is_v ? FPE_INFO_NDOF_V : FPE_INFO_NDOF_S);
  std::vector<double> tab(size_t(nq) * 4);
  std::vector<int32_t> c0(nq);
  if (nq > 0) {
    if (cudaMemcpy(tab.data(), P->d_arena + d.off_d + (is_v ? (deriv ? L.dB_v : L.B_v) : (deriv ? L.dB_s : L.B_s)),
                   tab.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
      return -1;
    if (cudaMemcpy(c0.data(), P->d_iarena + d.off_i + (is_v ? IL.c0_v : IL.c0_s), nq * sizeof(int32_t),
                   cudaMemcpyDeviceToHost) != cudaSuccess)
      return -1;
  }
  if (n_rows) *n_rows = nq;
  if (n_cols) *n_cols = nd;
  int64_t nnz = 0;
  if (indptr) indptr[0] = 0;
  for (int q = 0; q < nq; ++q) {
    for (int s = 0; s < 4; ++s) {
      const double v = tab[size_t(q) * 4 + s];
      const int col = c0[q] + s;
      if (v == 0.0 || col >= nd) continue;
      if (indices) indices[nnz] = col;
      if (data) data[nnz] = v;
      ++nnz;
    }
    if (indptr) indptr[q + 1] = int32_t(nnz);
  }
  return nnz;
}

void fpe_compute_free_vec(FpeVecResult* r) {
  if (r && r->data) std::free(r->data);
  if (r) *r = FpeVecResult{nullptr, 0};
}
void fpe_compute_free_vec2(FpeVec2Result* r) {
  if (!r) return;
  std::free(r->s_data);
  std::free(r->v_data);
  *r = FpeVec2Result{nullptr, 0, nullptr, 0};
}
void fpe_compute_free_grid_pts(FpeGridPtsResult* r) {
  if (!r) return;
  std::free(r->s_data);
  std::free(r->v_data);
  std::free(r->sw_data);
  std::free(r->vw_data);
  *r = FpeGridPtsResult{nullptr, 0, nullptr, 0, nullptr, nullptr};
}
void fpe_compute_free_mat(FpeMatResult* r) {
  if (r && r->data) std::free(r->data);
  if (r) *r = FpeMatResult{nullptr, 0, 0};
}
void fpe_compute_free_greeks(FpeGreeksResult* r) {
  if (!r) return;
  std::free(r->delta);
  std::free(r->gamma);
  std::free(r->vega);
  *r = FpeGreeksResult{nullptr, nullptr, nullptr, 0};
}
void fpe_compute_free_oneshot(FpeOneshotResult* r) {
  if (!r) return;
  std::free(r->price);
  std::free(r->delta);
  std::free(r->gamma);
  std::free(r->vega);
  *r = FpeOneshotResult{nullptr, nullptr, nullptr, nullptr, 0};
}

}  // extern "C"

// ==========================================================================
// Allocation-free pricing of one contract.
//
// Some callers cannot allocate device memory at pricing time: real-time and
// embedded hosts whose GPU memory budget is fixed at start-up, and plug-ins
// living inside another application that owns the device memory pool (its
// allocator may be exhausted or forbidden to them).  fpe_price_noalloc serves
// them from one file-scope static device array instead of per-call
// allocations; the caller passes the contract and receives the prices.
//
// The array (FPE_NOALLOC_SCRATCH_BYTES, 64 MiB) is held by every GPU that loads
// this library until the process exits.  Each device is set up on its first
// call, with that device current: the array's device address
// (cudaGetSymbolAddress), a stream of its own and the kernels' shared-memory
// opt-in.  Every call shares the array and it keeps the previous call's
// contents: the per-solve status words and the price slots are cleared at the
// start of each call, everything else is fully rewritten by the kernels.  Calls
// that overlap on the GPU (the same device, different streams or threads
// without ordering) race on the array and must be serialized by the caller.
// The call copies its results to host memory and waits for its stream, so it
// cannot run on a stream that is being captured into a graph: it checks that
// first and returns FPE_NOALLOC_ERR_CAPTURE without enqueuing anything.
// ==========================================================================
#define FPE_NOALLOC_SCRATCH_BYTES (64ull << 20)
#define FPE_NOALLOC_MAX_DEVICES 64
static __device__ __align__(256) unsigned char g_fpe_noalloc_scratch[FPE_NOALLOC_SCRATCH_BYTES];

struct NoallocDevice {
  unsigned char* base = nullptr;  // device address of the static array
  cudaStream_t stream = nullptr;  // used when the caller passes no stream
  int smem_optin = 0;
};

// Per-device set-up on the device's first call (the current device).
static NoallocDevice* noalloc_device(int device) {
  static NoallocDevice devs[FPE_NOALLOC_MAX_DEVICES];
  static std::mutex mu;
  if (device < 0 || device >= FPE_NOALLOC_MAX_DEVICES) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  NoallocDevice& D = devs[device];
  if (D.base) return &D;
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_fpe_noalloc_scratch) != cudaSuccess || !p) return nullptr;
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess) return nullptr;
  if (cudaFuncSetAttribute(fpe::k_setup, cudaFuncAttributeMaxDynamicSharedMemorySize, optin) != cudaSuccess ||
      cudaFuncSetAttribute(fpe::k_ic, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           optin - int(sizeof(fpe::IcSmem)) - 1024) != cudaSuccess ||
      fpe::radau_allow_smem<double>(optin) != cudaSuccess || fpe::radau_allow_smem<float>(optin) != cudaSuccess)
    return nullptr;
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
  D.stream = st;
  D.smem_optin = optin;
  D.base = static_cast<unsigned char*>(p);
  return &D;
}

extern "C" int32_t fpe_price_noalloc(const FpeContract* contract, const FpeBatchOptions* opt,
                                     double* prices, int32_t* status, void* cuda_stream) {
  if (!contract || !prices) return -1;
  const int nk = contract->n_strikes;
  if (nk <= 0 || nk > FPE_MAX_STRIKES || !contract->strikes) return FPE_NOALLOC_ERR_SIZE;
  if (opt && opt->greeks) return -1;
  if (cuda_stream) {  // a capturing stream would be invalidated by the host copies and the wait
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(static_cast<cudaStream_t>(cuda_stream), &cs) != cudaSuccess) return -1;
    if (cs != cudaStreamCaptureStatusNone) return FPE_NOALLOC_ERR_CAPTURE;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  NoallocDevice* ND = noalloc_device(dev);
  if (!ND) return -1;
  unsigned char* base = ND->base;
  cudaStream_t s = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : ND->stream;
  const Opts o = opts_from(opt, 50);

  // Pricing and its one or two device solves (in-out parity for knock-ins).
  Pricing p;
  p.kappa = contract->kappa; p.theta = contract->theta; p.sigma = contract->sigma;
  p.rho = contract->rho; p.r = contract->r; p.T = contract->T; p.S0 = contract->S0;
  p.V0 = contract->V0; p.barrier = contract->barrier;
  p.smin = contract->s_min >= 0.0 ? contract->s_min : 0.0;
  p.smax = contract->s_max > 0.0 ? contract->s_max : contract->S0 * 3.0;
  p.n_s = contract->n_s; p.n_v = contract->n_v; p.type = contract->option_type;
  p.strike_begin = 0;
  p.n_strikes = nk;
  p.valid = pricing_valid(p, contract->strikes) && p.n_s >= 4 && p.n_v >= 4 && p.n_s <= 256 &&
            p.n_v <= 256 && !(o.disc == 0 && grid_count_reference(o.num_insert, true) > 8192);
  if (!p.valid) {
    for (int j = 0; j < nk; ++j) {
      prices[j] = 0.0;
      if (status) status[j] = FPE_STATUS_INVALID;
    }
    return FPE_STATUS_INVALID;
  }
  FpeSolveDesc d[2];
  int nsolve = 1;
  const int ot = p.type;
  if (ot == 0 || ot == 1 || ot == 4 || ot == 5) {
    const bool call = ot % 2 == 0, down = ot <= 1;
    const Opts oki = knock_in_opts(o);
    d[0] = make_desc(p, call ? 8 : 9, 0.0, oki);
    d[1] = make_desc(p, (down ? 2 : 6) + (call ? 0 : 1), p.barrier, oki);
    nsolve = 2;
  } else {
    d[0] = make_desc(p, ot, p.barrier, o);
  }

  // Partition the static array: descriptors | strikes | prices | infos | arenas.
  const int esz = o.precision == 0 ? 8 : 4;
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  size_t off = 0;
  const size_t off_desc = off;
  off = up(off + 2 * sizeof(FpeSolveDesc));
  const size_t off_k = off;
  off = up(off + size_t(2) * nk * sizeof(double));
  const size_t off_p = off;
  off = up(off + size_t(2) * nk * sizeof(double));
  const size_t off_info = off;
  off = up(off + size_t(2) * FPE_INFO_COUNT * sizeof(int32_t));
  int64_t od = 0, oi = 0, of = 0;
  size_t smem_max = 0, smem_base = 0, ic = 0;
  for (int k = 0; k < nsolve; ++k) {
    resolve_solve_shape(d[k], o, esz, size_t(ND->smem_optin));
    d[k].strike_off = k * nk;
    d[k].off_d = od;
    d[k].off_i = oi;
    d[k].off_f = of;
    d[k].save_traj = 0;
    d[k].traj_cap = 0;
    d[k].off_traj = -1;
    od += fpe_dlayout(d[k]).total;
    oi += fpe_ilayout(d[k]).total;
    of += fpe_factor_bytes(d[k], esz, o.complex_mode);
    size_t b = 0;
    smem_max = std::max(smem_max, radau_smem_need(d[k], esz, o.complex_mode, &b));
    smem_base = std::max(smem_base, b);
    ic = std::max(ic, fpe_ic_admm_bytes(d[k].cap_dof_s, d[k].cap_dof_v));
  }
  const size_t off_d = off;
  off = up(off + size_t(od) * sizeof(double));
  const size_t off_i = off;
  off = up(off + size_t(oi) * sizeof(int32_t));
  const size_t off_f = off;
  off = up(off + size_t(of));
  if (off > FPE_NOALLOC_SCRATCH_BYTES) {
    for (int j = 0; j < nk; ++j) {
      prices[j] = 0.0;
      if (status) status[j] = FPE_STATUS_CAPACITY;
    }
    return FPE_NOALLOC_ERR_SIZE;  // the contract's grids need more than the static array
  }
  const size_t optin = size_t(ND->smem_optin);
  const int fac_global = smem_max > optin ? 1 : 0;
  const size_t radau_smem = fac_global ? smem_base : smem_max;
  const size_t ic_smem = ic <= optin - sizeof(fpe::IcSmem) - 1024 ? ic : 0;

  auto* g_desc = reinterpret_cast<FpeSolveDesc*>(base + off_desc);
  auto* g_k = reinterpret_cast<double*>(base + off_k);
  auto* g_p = reinterpret_cast<double*>(base + off_p);
  auto* g_info = reinterpret_cast<int32_t*>(base + off_info);
  auto* g_d = reinterpret_cast<double*>(base + off_d);
  auto* g_i = reinterpret_cast<int32_t*>(base + off_i);
  auto* g_f = reinterpret_cast<unsigned char*>(base + off_f);
  CK(cudaMemcpyAsync(g_desc, d, nsolve * sizeof(FpeSolveDesc), cudaMemcpyHostToDevice, s));
  for (int k = 0; k < nsolve; ++k)
    CK(cudaMemcpyAsync(g_k + k * nk, contract->strikes, nk * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(g_p, 0, size_t(2) * nk * sizeof(double), s));
  CK(cudaMemsetAsync(g_info, 0, size_t(2) * FPE_INFO_COUNT * sizeof(int32_t), s));
  const dim3 grid(nsolve), block(FPE_BLOCK);
  fpe::k_setup<<<grid, block, sizeof(fpe::SetupSmem), s>>>(g_desc, g_d, g_i, g_info);
  fpe::k_galerkin<<<grid, block, 0, s>>>(g_desc, g_d, g_i, g_info);
  fpe::k_ic<<<grid, block, ic_smem, s>>>(g_desc, g_d, g_i, g_info, ic_smem);
  const fpe::RadauConstants rk = fpe::radau_constants(o.radau_exact != 0);
  if (o.precision == 0) {
    fpe::RadauKernelArgs<double> a{g_desc, g_d, g_i, g_info, g_f, nullptr, 0, o.complex_mode,
                                   fac_global, rk.u1, rk.alph, rk.beta, rk.ti13, radau_smem,
                                   o.sweep_buffers ? o.sweep_buffers : FPE_SWEEP_BUFS};
    CK(fpe::launch_radau<double>(a, grid, dim3(FPE_RADAU_THREADS), radau_smem, s));
  } else {
    fpe::RadauKernelArgs<float> a{g_desc, g_d, g_i, g_info, g_f, nullptr, o.refine, o.complex_mode,
                                  fac_global, rk.u1, rk.alph, rk.beta, rk.ti13, radau_smem,
                                   o.sweep_buffers ? o.sweep_buffers : FPE_SWEEP_BUFS};
    CK(fpe::launch_radau<float>(a, grid, dim3(FPE_RADAU_THREADS), radau_smem, s));
  }
  fpe::k_payoff<<<grid, block, 0, s>>>(g_desc, g_d, g_i, g_info, g_k, g_p);
  CK(cudaGetLastError());
  double hp[2 * FPE_MAX_STRIKES];
  int32_t hi[2 * FPE_INFO_COUNT];
  CK(cudaMemcpyAsync(hp, g_p, size_t(nsolve) * nk * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(hi, g_info, size_t(nsolve) * FPE_INFO_COUNT * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  int worst = 0;
  for (int j = 0; j < nk; ++j) {
    double v = hp[j];
    int st = hi[FPE_INFO_STATUS];
    if (nsolve == 2) {
      v -= hp[nk + j];
      if (!st) st = hi[FPE_INFO_COUNT + FPE_INFO_STATUS];
    }
    prices[j] = v;
    if (status) status[j] = st;
    if (st && !worst) worst = st;
  }
  return worst;
}

// --------------------------------------------------------------------------
// Heston characteristic-function prices of Europeans (k_cf.cuh)
// --------------------------------------------------------------------------
namespace {

// 16-point Gauss-Legendre rule on [-1, 1]: Newton's method on the Legendre
// polynomial P16 (three-term recurrence) from the Chebyshev-like guesses
// cos(pi (i + 3/4) / (n + 1/2)); weights 2 / ((1 - x^2) P16'(x)^2).
const fpe::CfNodes& cf_nodes() {
  static fpe::CfNodes q;
  static std::once_flag once;
  std::call_once(once, [] {
    const int n = 16;
    for (int i = 0; i < n; ++i) {
      double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
      for (int it = 0; it < 100; ++it) {
        double p = 1.0, pm = 0.0;
        for (int k = 1; k <= n; ++k) {
          const double pk = ((2.0 * k - 1.0) * z * p - (k - 1.0) * pm) / k;
          pm = p;
          p = pk;
        }
        dp = n * (z * p - pm) / (z * z - 1.0);
        const double dz = p / dp;
        z -= dz;
        if (std::fabs(dz) < 1e-15) break;
      }
      q.x[i] = -z;
      q.w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
  });
  return q;
}

int launch_cf(const double* params, const double* strikes, const int32_t* put, int32_t n,
              double* out, cudaStream_t s) {
  const unsigned grid = unsigned((int64_t(n) + fpe::kCfWarps - 1) / fpe::kCfWarps);
  fpe::k_heston_cf<<<grid, 32 * fpe::kCfWarps, 0, s>>>(params, strikes, put, n, cf_nodes(), out);
  CK(cudaGetLastError());
  return 0;
}

}  // namespace

extern "C" int32_t fpe_heston_cf_batch(const double* params_dev, const double* strikes_dev,
                                       const int32_t* put_dev, int32_t n, double* prices_dev,
                                       void* cuda_stream) {
  if (n < 0) return -1;
  if (n == 0) return 0;
  if (!params_dev || !strikes_dev || !prices_dev) return -1;
  Context& C = ctx();
  if (!C.ok) return -1;
  cudaStream_t s = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : C.stream;
  return launch_cf(params_dev, strikes_dev, put_dev, n, prices_dev, s);
}

extern "C" int32_t fpe_heston_cf_price(const FpeContract* contracts, int32_t n, double* prices,
                                       int32_t* status) {
  if (n < 0 || (n > 0 && (!contracts || !prices))) return -1;
  Context& C = ctx();
  if (!C.ok) return -1;
  // one row per strike: 8 parameters, the strike and the put flag, packed
  // into one host buffer and copied with one transfer
  int64_t m = 0;
  for (int32_t c = 0; c < n; ++c) {
    if (contracts[c].n_strikes < 0 || (contracts[c].n_strikes > 0 && !contracts[c].strikes)) return -1;
    m += contracts[c].n_strikes;
  }
  if (m == 0) return 0;
  if (m > INT32_MAX) return -1;
  std::vector<int32_t> st(m, FPE_STATUS_OK);
  const size_t pbytes = size_t(m) * 9 * sizeof(double), bytes = pbytes + size_t(m) * sizeof(int32_t);
  std::vector<unsigned char> host(bytes);
  double* hp = reinterpret_cast<double*>(host.data());
  double* hk = hp + 8 * m;
  int32_t* hput = reinterpret_cast<int32_t*>(host.data() + pbytes);
  int64_t row = 0;
  for (int32_t c = 0; c < n; ++c) {
    const FpeContract& k = contracts[c];
    const bool euro = k.option_type == 8 || k.option_type == 9;
    const bool valid = k.kappa > 0 && k.theta > 0 && k.sigma > 0 && k.T > 0 && k.S0 > 0 &&
                       k.V0 >= 0 && k.rho >= -1 && k.rho <= 1 && std::isfinite(k.r);
    for (int32_t j = 0; j < k.n_strikes; ++j, ++row) {
      const double pr[8] = {k.kappa, k.theta, k.sigma, k.rho, k.r, k.T, k.S0, k.V0};
      std::memcpy(hp + 8 * row, pr, sizeof(pr));
      hk[row] = k.strikes[j];
      hput[row] = k.option_type == 9;
      if (!euro) {
        st[row] = FPE_STATUS_UNSUPPORTED;
        hp[8 * row] = -1.0;  // the kernel answers NaN for a non-positive kappa
      } else if (!valid || !(k.strikes[j] > 0.0)) {
        st[row] = FPE_STATUS_INVALID;
      }
    }
  }
  cudaStream_t s = C.stream;
  void* dev = nullptr;
  const size_t out_off = (bytes + 7) & ~size_t(7);
  CK(cudaMallocAsync(&dev, out_off + size_t(m) * sizeof(double), s));
  unsigned char* d = static_cast<unsigned char*>(dev);
  double* dout = reinterpret_cast<double*>(d + out_off);
  int rc = 0;
  if (cudaMemcpyAsync(d, host.data(), bytes, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      launch_cf(reinterpret_cast<double*>(d), reinterpret_cast<double*>(d) + 8 * m,
                reinterpret_cast<int32_t*>(d + pbytes), int32_t(m), dout, s) != 0 ||
      cudaMemcpyAsync(prices, dout, size_t(m) * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    rc = -1;
  cudaFreeAsync(dev, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) rc = -1;
  if (rc) return rc;
  int worst = 0;
  for (int64_t i = 0; i < m; ++i) {
    if (st[i] == FPE_STATUS_OK && !std::isfinite(prices[i])) st[i] = FPE_STATUS_NONFINITE;
    if (st[i] != FPE_STATUS_OK) prices[i] = std::nan("");
    if (status) status[i] = st[i];
    if (st[i] && !worst) worst = st[i];
  }
  return worst;
}

// --------------------------------------------------------------------------
// Terminal-density interpolation (k_interp.cuh)
// --------------------------------------------------------------------------
extern "C" int32_t fpe_pdf_interpolate(const double* s_points_dev, int32_t n_s, const double* v_points_dev,
                                       int32_t n_v, const double* pdf_dev, const double* s_dev,
                                       const double* v_dev, int32_t n, double* out_dev, void* cuda_stream) {
  if (n < 0 || n_s < 2 || n_v < 2) return -1;
  if (n == 0) return 0;
  if (!s_points_dev || !v_points_dev || !pdf_dev || !s_dev || !v_dev || !out_dev) return -1;
  Context& C = ctx();
  if (!C.ok) return -1;
  cudaStream_t st = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : C.stream;
  const int block = 256;
  const unsigned grid = unsigned((int64_t(n) + block - 1) / block);
  fpe::k_pdf_interp<<<grid, block, 0, st>>>(s_points_dev, n_s, v_points_dev, n_v, pdf_dev, s_dev, v_dev, n,
                                            out_dev);
  CK(cudaGetLastError());
  return 0;
}
