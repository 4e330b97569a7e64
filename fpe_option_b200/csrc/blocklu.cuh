// Block-banded LU of the Radau stage matrices, CTA-cooperative.
//
// E = a M + h K (real a) or (ALPH + i BETA) M + h K (complex shift), with
// M = As (x) Av and K = Ss (x) B1 + Tss (x) B2 + As (x) B3 + Ss^T (x) B4 in
// s-major order, is block-banded: nv x nv blocks (i, k), |i - k| <= 3.
// Block Gaussian elimination without inter-block pivoting (the pivot blocks
// are D-scaled and diagonally dominated by a M for the step sizes Radau uses;
// each pivot block is inverted by Gauss-Jordan with partial pivoting):
//   F[i][kk], kk = k - i + 3:
//     kk < 3 : L_{i,k} = E_{i,k} P_k^{-1}
//     kk = 3 : P_i^{-1}
//     kk > 3 : W_{i,k} = P_i^{-1} U_{i,k}
// A solve is then 2 ns dense block-GEMV steps (one barrier each):
//   forward  y_i = b_i - sum_k L_{i,i-k} y_{i-k},   z_i = P_i^{-1} y_i
//   backward x_i = z_i - sum_k W_{i,i+k} x_{i+k}
// Storage FT = float (FP32 factors, FP64 accumulation) or double; complex
// systems store interleaved (re, im) pairs.
#pragma once
#include "dev_common.cuh"

namespace fpe {

template <typename T>
struct Cx {
  T re, im;
};

template <typename T>
__device__ __forceinline__ Cx<T> cmk(T a, T b) {
  Cx<T> r;
  r.re = a;
  r.im = b;
  return r;
}

// Accumulator arithmetic (always FP64) over storage types.
__device__ __forceinline__ double acc_load(float v) { return double(v); }
__device__ __forceinline__ double acc_load(double v) { return v; }
__device__ __forceinline__ Cx<double> acc_load(Cx<float> v) { return cmk(double(v.re), double(v.im)); }
__device__ __forceinline__ Cx<double> acc_load(Cx<double> v) { return v; }

template <typename ET>
struct AccOf;
template <>
struct AccOf<float> { using T = double; };
template <>
struct AccOf<double> { using T = double; };
template <>
struct AccOf<Cx<float>> { using T = Cx<double>; };
template <>
struct AccOf<Cx<double>> { using T = Cx<double>; };

__device__ __forceinline__ void st_elem(float& d, double v) { d = float(v); }
__device__ __forceinline__ void st_elem(double& d, double v) { d = v; }
__device__ __forceinline__ void st_elem(Cx<float>& d, Cx<double> v) { d = cmk(float(v.re), float(v.im)); }
__device__ __forceinline__ void st_elem(Cx<double>& d, Cx<double> v) { d = v; }

template <typename T>
struct IsCx { static constexpr bool v = false; };
template <typename T>
struct IsCx<Cx<T>> { static constexpr bool v = true; };

__device__ __forceinline__ double azero(double) { return 0.0; }
__device__ __forceinline__ Cx<double> azero(Cx<double>) { return cmk(0.0, 0.0); }
__device__ __forceinline__ double aone(double) { return 1.0; }
__device__ __forceinline__ Cx<double> aone(Cx<double>) { return cmk(1.0, 0.0); }
// real / imaginary parts of an accumulator (imaginary of a real value is 0)
__device__ __forceinline__ double are(double a) { return a; }
__device__ __forceinline__ double are(Cx<double> a) { return a.re; }
__device__ __forceinline__ double aim(double) { return 0.0; }
__device__ __forceinline__ double aim(Cx<double> a) { return a.im; }
__device__ __forceinline__ void afma(double& a, double x, double y) { a = fma(x, y, a); }
__device__ __forceinline__ void afma(Cx<double>& a, Cx<double> x, Cx<double> y) {
  a.re = fma(x.re, y.re, fma(-x.im, y.im, a.re));
  a.im = fma(x.re, y.im, fma(x.im, y.re, a.im));
}
__device__ __forceinline__ double asub(double a, double b) { return a - b; }
__device__ __forceinline__ Cx<double> asub(Cx<double> a, Cx<double> b) { return cmk(a.re - b.re, a.im - b.im); }
__device__ __forceinline__ double amul(double a, double b) { return a * b; }
__device__ __forceinline__ Cx<double> amul(Cx<double> a, Cx<double> b) {
  return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
__device__ __forceinline__ double ainv(double a) { return a != 0.0 ? 1.0 / a : 0.0; }
__device__ __forceinline__ Cx<double> ainv(Cx<double> a) {
  const double d = a.re * a.re + a.im * a.im;
  return d != 0.0 ? cmk(a.re / d, -a.im / d) : cmk(0.0, 0.0);
}
__device__ __forceinline__ double amag(double a) { return fabs(a); }
__device__ __forceinline__ double amag(Cx<double> a) { return sqrt(a.re * a.re + a.im * a.im); }
__device__ __forceinline__ double shfl_down(double v, int o, int w) {
  return __shfl_down_sync(0xffffffffu, v, o, w);
}
__device__ __forceinline__ Cx<double> shfl_down(Cx<double> v, int o, int w) {
  return cmk(__shfl_down_sync(0xffffffffu, v.re, o, w), __shfl_down_sync(0xffffffffu, v.im, o, w));
}

// Operator factors held in shared memory (band 7, D-scaled).
struct OpFactors {
  int ns, nv;
  const double *As, *Ss, *Ts, *St;      // s: As, Ss~, Tss~, Ss~^T
  const double *Av, *B1, *B2, *B3, *B4; // v
};

template <typename ET>
struct BlockLU {
  ET* F;
  int ns, nv;
  __device__ __forceinline__ ET* blk(int i, int kk) const { return F + (size_t(i) * 7 + kk) * nv * nv; }
};

// E = (a_re + i a_im) M + h K into the block storage (a_im ignored for real ET).
template <typename ET>
__device__ void blu_assemble(const OpFactors& O, const BlockLU<ET>& L, double a_re, double a_im,
                             double h) {
  const int ns = O.ns, nv = O.nv;
  const size_t total = size_t(ns) * 7 * nv * nv;
  for (size_t e = threadIdx.x; e < total; e += blockDim.x) {
    const int jl = int(e % (nv * nv));
    const int ikk = int(e / (nv * nv));
    const int i = ikk / 7, kk = ikk - i * 7;
    const int j = jl / nv, l = jl - j * nv;
    const int k = i + kk - 3, dl = l - j + 3;
    double m = 0.0, kv = 0.0;
    if (k >= 0 && k < ns && dl >= 0 && dl < 7) {
      const int sb = i * 7 + kk, vb = j * 7 + dl;
      m = O.As[sb] * O.Av[vb];
      kv = O.Ss[sb] * O.B1[vb] + O.Ts[sb] * O.B2[vb] + O.As[sb] * O.B3[vb] + O.St[sb] * O.B4[vb];
    }
    if constexpr (!IsCx<ET>::v) {
      st_elem(L.F[e], a_re * m + h * kv);
    } else {
      st_elem(L.F[e], cmk(a_re * m + h * kv, a_im * m));
    }
  }
  __syncthreads();
}

// Factorization arithmetic type: the storage type (FP32 factors are computed
// in FP32, FP64 factors in FP64).
template <typename ET>
struct FacOf;
template <>
struct FacOf<float> { using T = float; };
template <>
struct FacOf<double> { using T = double; };
template <>
struct FacOf<Cx<float>> { using T = Cx<float>; };
template <>
struct FacOf<Cx<double>> { using T = Cx<double>; };

__device__ __forceinline__ float fzero(float) { return 0.f; }
__device__ __forceinline__ double fzero(double) { return 0.0; }
template <typename T>
__device__ __forceinline__ Cx<T> fzero(Cx<T>) { return cmk(T(0), T(0)); }
__device__ __forceinline__ float fone(float) { return 1.f; }
__device__ __forceinline__ double fone(double) { return 1.0; }
template <typename T>
__device__ __forceinline__ Cx<T> fone(Cx<T>) { return cmk(T(1), T(0)); }
__device__ __forceinline__ void ffma(float& a, float x, float y) { a = fmaf(x, y, a); }
__device__ __forceinline__ void ffma(double& a, double x, double y) { a = fma(x, y, a); }
template <typename T>
__device__ __forceinline__ void ffma(Cx<T>& a, Cx<T> x, Cx<T> y) {
  a.re = fma(x.re, y.re, fma(-x.im, y.im, a.re));
  a.im = fma(x.re, y.im, fma(x.im, y.re, a.im));
}
__device__ __forceinline__ float fsub(float a, float b) { return a - b; }
__device__ __forceinline__ double fsub(double a, double b) { return a - b; }
template <typename T>
__device__ __forceinline__ Cx<T> fsub(Cx<T> a, Cx<T> b) { return cmk(a.re - b.re, a.im - b.im); }
__device__ __forceinline__ float fmul(float a, float b) { return a * b; }
__device__ __forceinline__ double fmul(double a, double b) { return a * b; }
template <typename T>
__device__ __forceinline__ Cx<T> fmul(Cx<T> a, Cx<T> b) {
  return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
__device__ __forceinline__ float finv(float a) { return a != 0.f ? 1.f / a : 0.f; }
__device__ __forceinline__ double finv(double a) { return a != 0.0 ? 1.0 / a : 0.0; }
template <typename T>
__device__ __forceinline__ Cx<T> finv(Cx<T> a) {
  const T d = a.re * a.re + a.im * a.im;
  return d != T(0) ? cmk(a.re / d, -a.im / d) : cmk(T(0), T(0));
}
__device__ __forceinline__ double fmag(float a) { return fabs(double(a)); }
__device__ __forceinline__ double fmag(double a) { return fabs(a); }
template <typename T>
__device__ __forceinline__ double fmag(Cx<T> a) {
  return sqrt(double(a.re) * double(a.re) + double(a.im) * double(a.im));
}

// Shared scratch (in ET elements) needed by blu_factor for block size nv: the
// augmented pivot block [P | I] (row stride 2 nv + 1), the inverse P^-1, the
// staged E_{r,i} and U_{i,c} blocks and the computed L_{r,i} blocks, plus the
// Gauss-Jordan bookkeeping.
__host__ __device__ __forceinline__ int blu_smem_elems(int nv) {
  return nv * (2 * nv + 1) + 10 * nv * nv + 4 * nv + 16;
}

// 2 x 2 register tile of C = A B (nv x nv operands, row strides lda / ldb),
// rows j0, j0 + 1 and columns l0, l0 + 1 (guarded at odd edges).
template <typename ET>
__device__ __forceinline__ void tile2x2(const ET* A_, int lda, const ET* B_, int ldb, int nv, int j0,
                                        int l0, ET (&acc)[2][2]) {
  acc[0][0] = acc[0][1] = acc[1][0] = acc[1][1] = fzero(ET());
  const int j1 = min(j0 + 1, nv - 1), l1 = min(l0 + 1, nv - 1);
#pragma unroll 4
  for (int m = 0; m < nv; ++m) {
    const ET a0 = A_[j0 * lda + m], a1 = A_[j1 * lda + m];
    const ET b0 = B_[m * ldb + l0], b1 = B_[m * ldb + l1];
    ffma(acc[0][0], a0, b0);
    ffma(acc[0][1], a0, b1);
    ffma(acc[1][0], a1, b0);
    ffma(acc[1][1], a1, b1);
  }
}

// Shared (or global) factorization scratch of one system.
template <typename ET>
struct FacScratch {
  ET *aug, *Pi, *Eb, *Lb, *Ub;
  ET* fcol[2];   // elimination factors, double-buffered across columns
  int* prow_of;  // pivot row of each column
  int* used;     // row already pivotal
  int* ctl;      // [0], [1]: pivot row of the current / next column
  int nv, w1, nn;
  __device__ void init(ET* base, int nv_) {
    nv = nv_;
    w1 = 2 * nv + 1;
    nn = nv * nv;
    aug = base;
    Pi = aug + nv * w1;
    Eb = Pi + nn;
    Lb = Eb + 3 * nn;
    Ub = Lb + 3 * nn;
    fcol[0] = Ub + 3 * nn;
    fcol[1] = fcol[0] + nv;
    prow_of = reinterpret_cast<int*>(fcol[1] + nv);
    used = prow_of + nv;
    ctl = used + nv;
  }
};

// Scratch (ET elements) per system for block size nv.
__host__ __device__ __forceinline__ int blu_smem_elems_v2(int nv) {
  return nv * (2 * nv + 1) + 10 * nv * nv + 6 * nv + 16;
}

template <typename ET>
__device__ void fac_stage(const BlockLU<ET>& L, FacScratch<ET>& S, int i, int nr) {
  const int nv = S.nv, nn = S.nn, w1 = S.w1;
  const ET* P = L.blk(i, 3);
  for (int e = threadIdx.x; e < nv * 2 * nv; e += blockDim.x) {
    const int r = e / (2 * nv), c = e - r * (2 * nv);
    S.aug[r * w1 + c] = c < nv ? P[r * nv + c] : ((c - nv == r) ? fone(ET()) : fzero(ET()));
  }
  for (int e = threadIdx.x; e < nr * nn; e += blockDim.x) {
    const int cc = e / nn, jl = e - cc * nn;
    S.Ub[e] = L.blk(i, 4 + cc)[jl];
    S.Eb[e] = L.blk(i + 1 + cc, 2 - cc)[jl];
  }
  for (int r = threadIdx.x; r < nv; r += blockDim.x) S.used[r] = 0;
}

// Pivot selection for column c by warp `wsel` from the column values v[k]
// (rows lane + 32 k); writes the elimination factors and the pivot row.
template <typename ET>
__device__ __forceinline__ bool fac_pick(FacScratch<ET>& S, int c, const ET (&v)[2], int buf) {
  const int lane = threadIdx.x & 31, nv = S.nv;
  double best = -1.0;
  int bi = nv;
  for (int k = 0; k < 2; ++k) {
    const int r = lane + 32 * k;
    if (r < nv && !S.used[r]) {
      const double m = fmag(v[k]);
      if (m > best) {
        best = m;
        bi = r;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ob > best || (ob == best && oi < bi)) {
      best = ob;
      bi = oi;
    }
  }
  const int p = bi < nv ? bi : c;
  // broadcast the pivot value from its owning lane
  ET pv;
  {
    const int owner = p & 31, kk = p >> 5;
    ET mine = v[kk < 2 ? kk : 0];
    if constexpr (IsCx<ET>::v) {
      pv.re = __shfl_sync(0xffffffffu, mine.re, owner);
      pv.im = __shfl_sync(0xffffffffu, mine.im, owner);
    } else {
      pv = __shfl_sync(0xffffffffu, mine, owner);
    }
  }
  const ET inv = finv(pv);
  for (int k = 0; k < 2; ++k) {
    const int r = lane + 32 * k;
    if (r < nv) S.fcol[buf][r] = (r == p) ? fzero(ET()) : fmul(v[k], inv);
  }
  if (lane == 0) {
    S.ctl[buf] = p;
    S.used[p] = 1;
    S.prow_of[c] = p;
  }
  return best > 0.0;
}

// Gauss-Jordan elimination of column c (pivot row ctl[c&1]) by the CTA; warp
// `wsel` owns column c + 1, updates it first and picks its pivot (look-ahead),
// so each column costs one barrier.
template <typename ET>
__device__ bool fac_elim(FacScratch<ET>& S, int c, int wsel) {
  const int nv = S.nv, w1 = S.w1, buf = c & 1;
  const int p = S.ctl[buf];
  const ET* f = S.fcol[buf];
  const ET* prow = S.aug + p * w1;
  bool ok = true;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cn = c + 1;
  if (warp == wsel && cn < nv) {
    ET v[2];
    v[0] = v[1] = fzero(ET());
    for (int k = 0; k < 2; ++k) {
      const int r = lane + 32 * k;
      if (r >= nv) continue;
      ET& x = S.aug[r * w1 + cn];
      if (r != p) x = fsub(x, fmul(f[r], prow[cn]));
      v[k] = x;
    }
    ok = fac_pick<ET>(S, cn, v, buf ^ 1);
  }
  const int skip = cn < nv ? cn : -1;  // column already updated by the look-ahead warp
  for (int e = threadIdx.x; e < nv * 2 * nv; e += blockDim.x) {
    const int r = e / (2 * nv), l = e - r * (2 * nv);
    if (r == p || l == skip) continue;
    ET& x = S.aug[r * w1 + l];
    x = fsub(x, fmul(f[r], prow[l]));
  }
  return ok;
}

template <typename ET>
__device__ void fac_extract(const BlockLU<ET>& L, FacScratch<ET>& S, int i) {
  const int nv = S.nv, w1 = S.w1;
  for (int e = threadIdx.x; e < S.nn; e += blockDim.x) {
    const int c = e / nv, l = e - c * nv;
    const int p = S.prow_of[c];
    const ET v = fmul(S.aug[p * w1 + nv + l], finv(S.aug[p * w1 + c]));
    S.Pi[e] = v;
    L.blk(i, 3)[e] = v;
  }
}

// L_ri = E_ri P^-1 (shared), W_ic = P^-1 U_ic (global)
template <typename ET>
__device__ void fac_lw(const BlockLU<ET>& L, FacScratch<ET>& S, int i, int nr) {
  const int nv = S.nv, nn = S.nn, th = (nv + 1) / 2, ntile = th * th;
  for (int t = threadIdx.x; t < 2 * nr * ntile; t += blockDim.x) {
    const int job = t / ntile, tt = t - job * ntile;
    const int j0 = 2 * (tt / th), l0 = 2 * (tt - (tt / th) * th);
    ET acc[2][2];
    if (job < nr) {
      tile2x2<ET>(S.Eb + job * nn, nv, S.Pi, nv, nv, j0, l0, acc);
      ET* dst = S.Lb + job * nn;
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
          if (j0 + a < nv && l0 + b < nv) dst[(j0 + a) * nv + l0 + b] = acc[a][b];
    } else {
      const int cc = job - nr;
      tile2x2<ET>(S.Pi, nv, S.Ub + cc * nn, nv, nv, j0, l0, acc);
      ET* W = L.blk(i, 4 + cc);
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
          if (j0 + a < nv && l0 + b < nv) W[(j0 + a) * nv + l0 + b] = acc[a][b];
    }
  }
}

// L blocks out; E_rc -= L_ri U_ic
template <typename ET>
__device__ void fac_update(const BlockLU<ET>& L, FacScratch<ET>& S, int i, int nr) {
  const int nv = S.nv, nn = S.nn, th = (nv + 1) / 2, ntile = th * th;
  for (int e = threadIdx.x; e < nr * nn; e += blockDim.x) {
    const int rr = e / nn, jl = e - rr * nn;
    L.blk(i + 1 + rr, 2 - rr)[jl] = S.Lb[e];
  }
  for (int t = threadIdx.x; t < nr * nr * ntile; t += blockDim.x) {
    const int job = t / ntile, tt = t - job * ntile;
    const int j0 = 2 * (tt / th), l0 = 2 * (tt - (tt / th) * th);
    const int rr = job / nr, cc = job - rr * nr;
    ET acc[2][2];
    tile2x2<ET>(S.Lb + rr * nn, nv, S.Ub + cc * nn, nv, nv, j0, l0, acc);
    ET* E = L.blk(i + 1 + rr, cc - rr + 3);
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        if (j0 + a < nv && l0 + b < nv) {
          ET& x = E[(j0 + a) * nv + l0 + b];
          x = fsub(x, acc[a][b]);
        }
  }
}

// Factor the real stage matrix (and, when LC is given, the complex one in
// lockstep so both share every barrier).  scr_r / scr_c: scratch of
// blu_smem_elems_v2(nv) elements each.
template <typename FT>
__device__ bool blu_factor_pair(const BlockLU<FT>& LR, const BlockLU<Cx<FT>>* LC, FT* scr_r,
                                Cx<FT>* scr_c) {
  const int ns = LR.ns, nv = LR.nv;
  FacScratch<FT> SR;
  SR.init(scr_r, nv);
  FacScratch<Cx<FT>> SC;
  if (LC) SC.init(scr_c, nv);
  bool ok = true;
  const int warp = threadIdx.x >> 5;
  for (int i = 0; i < ns; ++i) {
    const int nr = min(i + 3, ns - 1) - i;
    fac_stage<FT>(LR, SR, i, nr);
    if (LC) fac_stage<Cx<FT>>(*LC, SC, i, nr);
    __syncthreads();
    // pivots of column 0 (warp 0: real, warp 1: complex)
    if (warp == 0) {
      FT v[2];
      v[0] = v[1] = fzero(FT());
      for (int k = 0; k < 2; ++k) {
        const int r = (threadIdx.x & 31) + 32 * k;
        if (r < nv) v[k] = SR.aug[r * SR.w1];
      }
      ok &= fac_pick<FT>(SR, 0, v, 0);
    } else if (warp == 1 && LC) {
      Cx<FT> v[2];
      v[0] = v[1] = fzero(Cx<FT>());
      for (int k = 0; k < 2; ++k) {
        const int r = (threadIdx.x & 31) + 32 * k;
        if (r < nv) v[k] = SC.aug[r * SC.w1];
      }
      ok &= fac_pick<Cx<FT>>(SC, 0, v, 0);
    }
    __syncthreads();
    for (int c = 0; c < nv; ++c) {
      ok &= fac_elim<FT>(SR, c, 0);
      if (LC) ok &= fac_elim<Cx<FT>>(SC, c, 1);
      __syncthreads();
    }
    fac_extract<FT>(LR, SR, i);
    if (LC) fac_extract<Cx<FT>>(*LC, SC, i);
    __syncthreads();
    if (nr > 0) {
      fac_lw<FT>(LR, SR, i, nr);
      if (LC) fac_lw<Cx<FT>>(*LC, SC, i, nr);
      __syncthreads();
      fac_update<FT>(LR, SR, i, nr);
      if (LC) fac_update<Cx<FT>>(*LC, SC, i, nr);
      __syncthreads();
    }
  }
  return ok;
}

// Right-hand sides of one fused solve: up to two real vectors on the real
// factor and one complex vector (re, im arrays) on the complex factor.
template <typename FT>
struct SolveSet {
  const BlockLU<FT>* R;
  const BlockLU<Cx<FT>>* Cf;
  double* xr[2];   // in: b, out: x
  double* zr[2];   // scratch N
  int nr;
  double* xc_re;
  double* xc_im;
  double* zc_re;
  double* zc_im;
  int nc;  // 0 or 1
};

template <typename ET, typename A>
__device__ __forceinline__ A grp_dot(const ET* row, const double* xre, const double* xim, int nv, int gl, int G);

template <>
__device__ __forceinline__ double grp_dot<float, double>(const float* row, const double* x, const double*, int nv,
                                                         int gl, int G) {
  double a = 0.0;
  for (int m = gl; m < nv; m += G) a = fma(double(row[m]), x[m], a);
  return a;
}
template <>
__device__ __forceinline__ double grp_dot<double, double>(const double* row, const double* x, const double*,
                                                          int nv, int gl, int G) {
  double a = 0.0;
  for (int m = gl; m < nv; m += G) a = fma(row[m], x[m], a);
  return a;
}
template <>
__device__ __forceinline__ Cx<double> grp_dot<Cx<float>, Cx<double>>(const Cx<float>* row, const double* xr,
                                                                      const double* xi, int nv, int gl, int G) {
  Cx<double> a = cmk(0.0, 0.0);
  for (int m = gl; m < nv; m += G) afma(a, acc_load(row[m]), cmk(xr[m], xi[m]));
  return a;
}
template <>
__device__ __forceinline__ Cx<double> grp_dot<Cx<double>, Cx<double>>(const Cx<double>* row, const double* xr,
                                                                       const double* xi, int nv, int gl, int G) {
  Cx<double> a = cmk(0.0, 0.0);
  for (int m = gl; m < nv; m += G) afma(a, row[m], cmk(xr[m], xi[m]));
  return a;
}

// Fused block solve of all right-hand sides in S (2 ns + 1 barriers).  Thread
// groups of G lanes own one row of one system; every lane executes the same
// shuffle reductions (real systems carry a zero imaginary part).
template <typename FT>
__device__ void blu_solve(const SolveSet<FT>& S) {
  const int ns = S.R ? S.R->ns : S.Cf->ns;
  const int nv = S.R ? S.R->nv : S.Cf->nv;
  const int rows = (S.nr + S.nc) * nv;
  int G = 32;
  while (G > 1 && rows * G > int(blockDim.x)) G >>= 1;
  const int grp = threadIdx.x / G, gl = threadIdx.x - grp * G;
  const bool act = grp < rows;
  const int sys = act ? grp / nv : 0;  // 0..nr-1 real, nr complex
  const int j = act ? grp - sys * nv : 0;
  const bool is_c = act && sys >= S.nr;
  const bool is_r = act && sys < S.nr;
  auto reduce4 = [&](double& a, double& b, double& c, double& d) {
    for (int o = G >> 1; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o, G);
      b += __shfl_down_sync(0xffffffffu, b, o, G);
      c += __shfl_down_sync(0xffffffffu, c, o, G);
      d += __shfl_down_sync(0xffffffffu, d, o, G);
    }
  };
  // forward (+ z of the previous block row)
  for (int i = 0; i <= ns; ++i) {
    double ar = 0.0, ai = 0.0, zr = 0.0, zi = 0.0;
    if (is_r) {
      const BlockLU<FT>& L = *S.R;
      const double* x = S.xr[sys];
      if (i < ns)
        for (int k = 1; k <= 3 && i - k >= 0; ++k)
          ar += grp_dot<FT, double>(L.blk(i, 3 - k) + j * nv, x + (i - k) * nv, nullptr, nv, gl, G);
      if (i > 0) zr = grp_dot<FT, double>(L.blk(i - 1, 3) + j * nv, x + (i - 1) * nv, nullptr, nv, gl, G);
    } else if (is_c) {
      const BlockLU<Cx<FT>>& L = *S.Cf;
      if (i < ns)
        for (int k = 1; k <= 3 && i - k >= 0; ++k) {
          const Cx<double> d = grp_dot<Cx<FT>, Cx<double>>(L.blk(i, 3 - k) + j * nv, S.xc_re + (i - k) * nv,
                                                           S.xc_im + (i - k) * nv, nv, gl, G);
          ar += d.re;
          ai += d.im;
        }
      if (i > 0) {
        const Cx<double> d = grp_dot<Cx<FT>, Cx<double>>(L.blk(i - 1, 3) + j * nv, S.xc_re + (i - 1) * nv,
                                                         S.xc_im + (i - 1) * nv, nv, gl, G);
        zr = d.re;
        zi = d.im;
      }
    }
    reduce4(ar, ai, zr, zi);
    if (gl == 0) {
      if (is_r) {
        if (i > 0 && i < ns) S.xr[sys][i * nv + j] -= ar;
        if (i > 0) S.zr[sys][(i - 1) * nv + j] = zr;
      } else if (is_c) {
        if (i > 0 && i < ns) {
          S.xc_re[i * nv + j] -= ar;
          S.xc_im[i * nv + j] -= ai;
        }
        if (i > 0) {
          S.zc_re[(i - 1) * nv + j] = zr;
          S.zc_im[(i - 1) * nv + j] = zi;
        }
      }
    }
    __syncthreads();
  }
  // backward: x_i = z_i - sum_k W_{i,i+k} x_{i+k}
  for (int i = ns - 1; i >= 0; --i) {
    double ar = 0.0, ai = 0.0, d0 = 0.0, d1 = 0.0;
    if (is_r) {
      const BlockLU<FT>& L = *S.R;
      const double* x = S.xr[sys];
      for (int k = 1; k <= 3 && i + k < ns; ++k)
        ar += grp_dot<FT, double>(L.blk(i, 3 + k) + j * nv, x + (i + k) * nv, nullptr, nv, gl, G);
    } else if (is_c) {
      const BlockLU<Cx<FT>>& L = *S.Cf;
      for (int k = 1; k <= 3 && i + k < ns; ++k) {
        const Cx<double> d = grp_dot<Cx<FT>, Cx<double>>(L.blk(i, 3 + k) + j * nv, S.xc_re + (i + k) * nv,
                                                         S.xc_im + (i + k) * nv, nv, gl, G);
        ar += d.re;
        ai += d.im;
      }
    }
    reduce4(ar, ai, d0, d1);
    if (gl == 0) {
      if (is_r) {
        S.xr[sys][i * nv + j] = S.zr[sys][i * nv + j] - ar;
      } else if (is_c) {
        S.xc_re[i * nv + j] = S.zc_re[i * nv + j] - ar;
        S.xc_im[i * nv + j] = S.zc_im[i * nv + j] - ai;
      }
    }
    __syncthreads();
  }
}

}  // namespace fpe
