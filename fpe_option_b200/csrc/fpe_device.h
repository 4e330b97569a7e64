// Shared host/device layout of one batched Fokker-Planck solve.
//
// A batch is a list of independent solves.  Each solve owns one slot in three
// arenas (FP64 data, int32 data, stage-system factors) whose offsets the host
// computes from per-solve capacity bounds.  All kernels run one CTA per solve.
#pragma once
#include <stdint.h>

#define FPE_BLOCK 256
// Threads of the persistent Radau kernel's CTA (one CTA per solve).
#ifndef FPE_RADAU_THREADS
#define FPE_RADAU_THREADS 256
#endif
#define FPE_MAX_STRIKES 1024
#define FPE_MAX_NDOF_V 64      // block size of the block-banded stage LU
#define FPE_MAX_NDOF_S 160
#define FPE_GMRES_M 10

// Status word per solve (0 = ok).
enum FpeStatus : int32_t {
  FPE_OK = 0,
  FPE_ERR_CAPACITY = 1,      // a discretization array exceeded its bound
  FPE_ERR_UNSUPPORTED = 2,   // n_dof_v above the block-LU limit
  FPE_ERR_SINGULAR = 3,      // zero pivot in a diagonal block
  FPE_ERR_MAX_STEPS = 4,     // radau.mojo:257-263
  FPE_ERR_STEP_UNDERFLOW = 5,// radau.mojo:274-281, :458-464
  FPE_ERR_NONFINITE = 6,
  FPE_ERR_TIMEOUT = 7,       // a bounded wait on an asynchronous copy gave up
};

// Per-solve counters written by the kernels (int32 arena, FPE_INFO_* slots).
enum FpeInfo {
  FPE_INFO_STATUS = 0,
  FPE_INFO_NKNOT_S, FPE_INFO_NKNOT_V, FPE_INFO_NGRID_S, FPE_INFO_NGRID_V,
  FPE_INFO_NQ_S, FPE_INFO_NQ_V, FPE_INFO_NDOF_S, FPE_INFO_NDOF_V,
  FPE_INFO_ACCEPTED, FPE_INFO_REJECTED, FPE_INFO_NEWTON, FPE_INFO_GMRES, FPE_INFO_LU,
  FPE_INFO_ADMM, FPE_INFO_PASS_REAL, FPE_INFO_NSAVED, FPE_INFO_PASS_CPLX,
  // SM clock cycles / 1024 spent in the Radau kernel phases (thread 0's view)
  FPE_INFO_T_FACTOR, FPE_INFO_T_SOLVE, FPE_INFO_T_KRON, FPE_INFO_T_TOTAL,
  FPE_INFO_T_FGJ,    // inside T_FACTOR: pivot-block Gauss-Jordan (kilocycles)
  FPE_INFO_T_FGEMM,  // inside T_FACTOR: L / W products and Schur updates (kilocycles)
  FPE_INFO_T_SWAIT,  // inside T_SOLVE: waits for the staged sweeps' bulk copies (kilocycles)
  // inside T_FGJ, each role's own work before the phase's closing barrier
  // (kilocycles): the real pivot inverse (warp 0), the complex one (warp 1)
  // and the other Schur updates (warp 2)
  FPE_INFO_T_GJ_REAL, FPE_INFO_T_GJ_CPLX, FPE_INFO_T_SCHUR,
  FPE_INFO_T_FASM,    // inside T_FACTOR: stage-matrix assembly (kilocycles)
  FPE_INFO_T_FSTAGE,  // inside T_FACTOR: staging of each block row and the pivot-inverse extraction
  // inside T_SOLVE (kilocycles): a stage's work after its copies landed, up
  // to the stage barrier, for thread 0 (a real row) and for the first thread
  // of the complex rows; and thread 0's wait at the stage barrier
  FPE_INFO_T_SREAL, FPE_INFO_T_SCPLX, FPE_INFO_T_SBAR,
  FPE_INFO_COUNT = 40
};

struct FpeSolveDesc {
  // Heston parameters (already revised for the barrier domain)
  double kappa, theta, sigma, rho, r, T, S0, V0;
  double smin, smax, vmin, vmax;
  double barrier;
  double rtol, atol;
  double max_step;       // <= 0: T / 5 (the reference Pricer)
  double first_step;     // 0: 1e-6 (Pricer); < 0: the Radau solver's estimate
  double ic_sigma_s, ic_sigma_v;
  int32_t type;          // 0..9; knock-ins are split into two solves by the host
  int32_t n_s, n_v;      // knot-count inputs
  int32_t left_neu, right_neu;
  int32_t disc;          // 0 reference, 1 config
  int32_t price_rule;    // 1: calibration-objective integration (reference disc)
  int32_t num_insert;
  int32_t ic_sub;
  int32_t strike_off, n_strikes;
  int32_t save_traj;     // keep every accepted step (stepwise API)
  int32_t traj_cap;      // max saved states
  int32_t max_steps;     // accepted-step cap (radau.mojo:257-263: 100000)
  int32_t blk_split;     // stage-LU block size nv / blk_split (1 or 2; see fpe_blk_split)
  int32_t sweep_bufs;    // stage buffers of the staged sweeps (2 .. 4; 0: the launch's default)
  int32_t pad1;
  int64_t stage_wait;    // SM cycles a staged sweep waits for its copies (<= 0: ~1 s)
  // capacities
  int32_t cap_knot_s, cap_knot_v, cap_grid_s, cap_grid_v, cap_q_s, cap_q_v;
  int32_t cap_dof_s, cap_dof_v;
  // arena offsets (elements)
  int64_t off_d;         // double arena
  int64_t off_i;         // int32 arena
  int64_t off_f;         // factor arena (bytes)
  int64_t off_traj;      // trajectory arena (doubles), -1 when not saved
};

// Offsets of the sub-arrays inside one solve's double slot.  Computed
// identically on host and device from the descriptor capacities.
struct FpeDLayout {
  int64_t knot_s, knot_v, grid_s, grid_v;
  int64_t qx_s, qw_s, qp_s, qx_v, qw_v, qp_v;      // nodes: normalized, weight, physical
  int64_t B_s, dB_s, B_v, dB_v;                     // 4 values per node
  int64_t fac_s, fac_v;                             // raw 1-D Galerkin factors
  int64_t op_s, op_v, D_s, D_v, m_s, m_v;           // scaled operator factors
  int64_t proj, q0, y, qT;                          // vectors of length N
  int64_t fsc;                                      // factorization scratch (global fallback)
  int64_t work;                                     // Radau/GMRES/ADMM work area
  int64_t total;
};

struct FpeILayout {
  int64_t info, c0_s, c0_v, rng_s, rng_v, total;
};

// Number of raw 1-D factors per axis and their order.
//   s: 0 Ns = Bs^T W Bs, 1 Ss = dBs^T W s Bs, 2 Tss = dBs^T W s^2 dBs
//   v: 0 Nv, 1 V2 = Bv^T W v Bv, 2 V3 = Bv^T W v dBv, 3 V4 = dBv^T W Bv,
//      4 V5 = dBv^T W v Bv, 5 V6 = dBv^T W v dBv
#define FPE_NFAC_S 3
#define FPE_NFAC_V 6
// Scaled operator factors (band 7, D-scaled):
//   s: 0 As, 1 Ss~, 2 Tss~, 3 Ss~^T        v: 0 Av, 1 B1, 2 B2, 3 B3, 4 B4
#define FPE_NOP_S 4
#define FPE_NOP_V 5
#define FPE_WORK_VECS 80   // N-length FP64 work vectors per solve

#ifdef __CUDACC__
#define FPE_HD __host__ __device__ __forceinline__
#else
#define FPE_HD inline
#endif

// Block structure of the stage LU for nv v-dofs: blocks of b = nv / m with
// bw = 4 m - 1 off-diagonal blocks per side (m = 1: one s-coupling per block,
// bw = 3; m = 2: half-width blocks, bw = 7).  m = 2 needs an even nv.
FPE_HD int fpe_blk_split(int requested, int nv) { return (requested == 2 && nv % 2 == 0 && nv >= 8) ? 2 : 1; }
FPE_HD int fpe_blk_bw(int m) { return 4 * m - 1; }

// Stage-factorization scratch of one system, in elements, for block size b
// and bw off-diagonal blocks: the pivot block's Gauss-Jordan array
// b x (b + 1), then blocks padded to p = b rounded up to 4, a whole number
// of register tiles (row-major p x p, transposed p x (p + 4)): P^-1 both
// ways, bw transposed E and L blocks, bw U blocks, and the pivot bookkeeping
// (with room to spare).
FPE_HD int fpe_fac_nvp(int nv) { return (nv + 3) & ~3; }
// Element stride between the b x b blocks of a stored stage factor: b^2
// rounded up to 4, so every block starts and ends on a 16-byte boundary and
// moves with one bulk copy.
FPE_HD int fpe_block_stride(int b) { return (b * b + 3) & ~3; }
FPE_HD int fpe_fac_scratch_elems(int b, int bw = 3) {
  const int p = fpe_fac_nvp(b), t = p + 4;
  const int aug = (b * (b + 1) + 3) & ~3;
  return aug + p * p + p * t + bw * p * t + bw * p * t + bw * p * p + 3 * p + (3 * p + 4);
}

// Shared memory of the IC projection's ADMM (bytes): eigenvector matrices
// Vs (nds x (nds + 2)), Vv and Vv^T (ndv^2 each), the iterates, lam and q (N
// each) and the intermediate (nds x (ndv + 2)), every section rounded to an
// even number of doubles.
// Vs and the products' intermediate have their rows padded by two doubles
// (strides nds + 2 and ndv + 2), so the row-wise operand loads of a warp's
// tiles fall on different banks.
FPE_HD size_t fpe_ic_admm_bytes(int nds, int ndv) {
  auto ev = [](size_t n) { return (n + 1) & ~size_t(1); };
  const size_t N = size_t(nds) * ndv;
  return (ev(size_t(nds) * (nds + 2)) + 2 * ev(size_t(ndv) * ndv) + 6 * ev(N) + ev(size_t(nds) * (ndv + 2))) *
         sizeof(double);
}

FPE_HD FpeDLayout fpe_dlayout(const FpeSolveDesc& d) {
  FpeDLayout L;
  int64_t o = 0;
  auto take = [&](int64_t n) {
    int64_t r = o;
    o += (n + 7) & ~int64_t(7);
    return r;
  };
  int64_t N = int64_t(d.cap_dof_s) * d.cap_dof_v;
  L.knot_s = take(d.cap_knot_s);
  L.knot_v = take(d.cap_knot_v);
  L.grid_s = take(d.cap_grid_s);
  L.grid_v = take(d.cap_grid_v);
  L.qx_s = take(d.cap_q_s);
  L.qw_s = take(d.cap_q_s);
  L.qp_s = take(d.cap_q_s);
  L.qx_v = take(d.cap_q_v);
  L.qw_v = take(d.cap_q_v);
  L.qp_v = take(d.cap_q_v);
  L.B_s = take(4 * int64_t(d.cap_q_s));
  L.dB_s = take(4 * int64_t(d.cap_q_s));
  L.B_v = take(4 * int64_t(d.cap_q_v));
  L.dB_v = take(4 * int64_t(d.cap_q_v));
  L.fac_s = take(int64_t(FPE_NFAC_S) * d.cap_dof_s * 7);
  L.fac_v = take(int64_t(FPE_NFAC_V) * d.cap_dof_v * 7);
  L.op_s = take(int64_t(FPE_NOP_S) * d.cap_dof_s * 7);
  L.op_v = take(int64_t(FPE_NOP_V) * d.cap_dof_v * 7);
  L.D_s = take(d.cap_dof_s);
  L.D_v = take(d.cap_dof_v);
  L.m_s = take(d.cap_dof_s);
  L.m_v = take(d.cap_dof_v);
  L.proj = take(N);
  L.q0 = take(N);
  L.y = take(N);
  L.qT = take(N);
  // FP64 worst case of the real + complex factor scratch (elements of 8 and
  // 16 bytes) plus the 16-byte alignment of the complex part
  L.fsc = take(3 * int64_t(fpe_fac_scratch_elems(d.cap_dof_v)) + 8);
  int64_t dense = int64_t(d.cap_dof_s) * d.cap_dof_s + int64_t(d.cap_dof_v) * d.cap_dof_v;
  L.work = take(int64_t(FPE_WORK_VECS) * N + 4 * dense + 256);
  L.total = o;
  return L;
}

FPE_HD FpeILayout fpe_ilayout(const FpeSolveDesc& d) {
  FpeILayout L;
  int64_t o = 0;
  auto take = [&](int64_t n) {
    int64_t r = o;
    o += (n + 3) & ~int64_t(3);
    return r;
  };
  L.info = take(FPE_INFO_COUNT);
  L.c0_s = take(d.cap_q_s);
  L.c0_v = take(d.cap_q_v);
  L.rng_s = take(2 * int64_t(d.cap_dof_s));
  L.rng_v = take(2 * int64_t(d.cap_dof_v));
  L.total = o;
  return L;
}

// Bytes of stage-system factor storage: one real block-banded LU (ns m block
// rows x 2 bw + 1 blocks of b x b) of element size esz, plus the same for the
// complex system when requested (2 * esz per entry).  The kernel picks the
// block split from the solve's actual nv; the size covers both splits.
FPE_HD int64_t fpe_factor_bytes(const FpeSolveDesc& d, int esz, int with_complex) {
  int64_t blocks = int64_t(d.cap_dof_s) * 7 * fpe_block_stride(d.cap_dof_v);
  if (d.blk_split == 2) {
    const int64_t b2 = int64_t(d.cap_dof_s) * 2 * 15 * fpe_block_stride((d.cap_dof_v + 1) / 2);
    if (b2 > blocks) blocks = b2;
  }
  int64_t b = blocks * esz;
  if (with_complex) b += blocks * 2 * esz;
  return (b + 255) & ~int64_t(255);
}
