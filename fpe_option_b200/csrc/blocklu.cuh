// Block-banded LU of the Radau stage matrices, CTA-cooperative.
//
// E = a M + h K (real a) or (ALPH + i BETA) M + h K (complex shift), with
// M = As (x) Av and K = Ss (x) B1 + Tss (x) B2 + As (x) B3 + Ss^T (x) B4 in
// s-major order (index i nv + j), is banded: entries couple s-dofs |i - k| <= 3
// and v-dofs |j - l| <= 3.  It is stored block-banded with block size
// b = nv / m (m = 1 or 2): nb = ns m block rows, bw = 4 m - 1 off-diagonal
// blocks on each side (m = 1: the nv x nv blocks of one s-coupling, bw = 3;
// m = 2: half-width blocks, bw = 7).  Both hold the same band (4 nv wide) and
// cost the same flops; smaller blocks need less scratch and shorten each
// pivot inverse, larger ones need fewer sequential steps.
// Block Gaussian elimination without inter-block pivoting (the pivot blocks
// are D-scaled and diagonally dominated by a M for the step sizes Radau uses;
// each pivot block is inverted by Gauss-Jordan with partial pivoting):
//   F[i][kk], kk = k - i + bw:
//     kk < bw : L_{i,k} = E_{i,k} P_k^{-1}
//     kk = bw : P_i^{-1}
//     kk > bw : W_{i,k} = P_i^{-1} U_{i,k}
// A solve is then 2 nb dense block-GEMV steps (one barrier each):
//   forward  y_i = b_i - sum_k L_{i,i-k} y_{i-k},   z_i = P_i^{-1} y_i
//   backward x_i = z_i - sum_k W_{i,i+k} x_{i+k}
// Storage FT = float (FP32 factors, FP64 accumulation) or double; complex
// systems store interleaved (re, im) pairs.
#pragma once
#include "dev_common.cuh"
#include "bulk_pipe.cuh"

// The dynamic shared memory of the launch.  Pointers formed from it keep
// their shared address space through inlining, so their loads are LDS; a
// pointer carried through a struct member is generic and its loads take the
// slower generic path (long scoreboard).
extern __shared__ __align__(16) unsigned char fpe_dsmem[];

__device__ __forceinline__ uint32_t dsmem_offset(const void* p) {
  return uint32_t(reinterpret_cast<const unsigned char*>(p) - fpe_dsmem);
}

// The pivot-block inverse used by the factorization (fac_gj: registers for FP32
// blocks where it can; fac_gj_warp: shared-memory rows).
#ifndef FPE_GJ
#define FPE_GJ fac_gj
#endif

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

// Block-banded storage of one stage matrix: block row i holds 2 bw + 1 blocks
// of b x b, kk = 0 .. 2 bw for block columns i - bw .. i + bw, each at a
// stride of fpe_block_stride(b) elements.  Before and during the
// factorization a block is row-major; the final factor blocks (L in kk < bw,
// P^-1 in kk = bw, W = P^-1 U in kk > bw) are stored transposed (element
// (j, m) at m b + j), so that the sweeps read each block column-wise with one
// output row per thread.
template <typename ET>
struct BlockLU {
  ET* F;
  int nb;  // block rows (ns m)
  int b;   // block size (nv / m)
  int bs;  // element stride between blocks
  int bw;  // off-diagonal blocks per side (4 m - 1)
  int nv;  // v-dofs of the grid
  __device__ __forceinline__ ET* blk(int i, int kk) const { return F + (size_t(i) * (2 * bw + 1) + kk) * bs; }
};

// Four consecutive elements to a 16-byte-aligned address with 16-byte stores.
__device__ __forceinline__ void store4(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void store4(double* p, const double (&v)[4]) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void store4(Cx<float>* p, const Cx<float> (&v)[4]) {
  reinterpret_cast<float4*>(p)[0] = make_float4(v[0].re, v[0].im, v[1].re, v[1].im);
  reinterpret_cast<float4*>(p)[1] = make_float4(v[2].re, v[2].im, v[3].re, v[3].im);
}
__device__ __forceinline__ void store4(Cx<double>* p, const Cx<double> (&v)[4]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) reinterpret_cast<double2*>(p)[k] = make_double2(v[k].re, v[k].im);
}

// E_r = a_r M + h K into LR and, when cplx, E_c = (c_re + i c_im) M + h K into
// LC, in one pass over the blocks (both need the same entries of M and K).
// Compiled as a function of its own: the operator factors (shared memory) and
// the block descriptions arrive by value and are read into registers once, so
// that no read in the loop goes to the kernel's stack frame (whose slots the
// compiler must reload after every store through a global pointer).  The
// blocks of a block row whose column lies outside the matrix (k < 0 or
// k >= nb) are never read, by the factorization or by the sweeps, and are not
// written; neither is the padding after a block's b^2 entries.  Rows and
// columns inside a block come from the exact float reciprocal (arguments
// below 2^16), not from integer divisions.
template <typename FT>
__device__ __noinline__ void blu_assemble_pair(OpFactors O, BlockLU<FT> LR, BlockLU<Cx<FT>> LC, bool cplx,
                                               double a_r, double c_re, double c_im, double h) {
  // the factors as shared-memory pointers (they live in the launch's dynamic
  // shared memory), so that their loads are LDS
  auto sh = [](const double* p) { return reinterpret_cast<const double*>(fpe_dsmem + dsmem_offset(p)); };
  const double *As = sh(O.As), *Ss = sh(O.Ss), *Ts = sh(O.Ts), *St = sh(O.St);
  const double *Av = sh(O.Av), *B1 = sh(O.B1), *B2 = sh(O.B2), *B3 = sh(O.B3), *B4 = sh(O.B4);
  FT* const FR = LR.F;
  Cx<FT>* const FC = LC.F;
  const int nb = LR.nb, b = LR.b, nv = O.nv, bs = LR.bs, bw = LR.bw, w = 2 * bw + 1, nn = b * b;
  const float rb = 1.0f / float(b), rnv = 1.0f / float(nv);
  if (b == nv && (nv & 3) == 0) {
    // nv x nv blocks, nv a multiple of 4: one s-coupling per block, rows and
    // columns are v-dofs, nonzero only on the 7 diagonals |j - l| <= 3.  A
    // thread fills 4 consecutive entries of a row (16-byte-aligned vector
    // stores) and computes only those on the band.  Work items q run over
    // (block, chunk) pairs.
    const int cpr = nv >> 2, nch = nn >> 2;
    const float rcpr = 1.0f / float(cpr);
    const int total = nb * w * nch;
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
      const int blk = q / nch, ch = q - blk * nch;
      const int i = blk / w, kk = blk - w * i;
      const int k = i + kk - bw;
      if (k < 0 || k >= nb) continue;
      const int j = int((float(ch) + 0.5f) * rcpr), l0 = (ch - j * cpr) << 2;
      const int sb = i * 7 + kk - bw + 3;
      FT vr[4];
      Cx<FT> vc[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int dl = l0 + u - j + 3;
        double m = 0.0, kv = 0.0;
        if (dl >= 0 && dl < 7) {
          const int vb = j * 7 + dl;
          const double as = As[sb];
          m = as * Av[vb];
          kv = Ss[sb] * B1[vb] + Ts[sb] * B2[vb] + as * B3[vb] + St[sb] * B4[vb];
        }
        vr[u] = FT(a_r * m + h * kv);
        vc[u] = cmk(FT(c_re * m + h * kv), FT(c_im * m));
      }
      const size_t off = size_t(blk) * bs + size_t(j) * nv + l0;
      store4(FR + off, vr);
      if (cplx) store4(FC + off, vc);
    }
  } else {
    // general blocks (b = nv / m): entry (jj, ll) of block (i, kk) is the
    // coupling of global row r = i b + jj = si nv + vj and column
    // c = k b + ll = sk nv + vl
    const int total = nb * w * nn;
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
      const int blk = q / nn, e = q - blk * nn;
      const int i = blk / w, kk = blk - w * i;
      const int k = i + kk - bw;
      if (k < 0 || k >= nb) continue;
      const int jj = int((float(e) + 0.5f) * rb), ll = e - jj * b;
      const int r = i * b + jj, c = k * b + ll;
      const int si = int((float(r) + 0.5f) * rnv), vj = r - si * nv;
      const int sk = int((float(c) + 0.5f) * rnv), vl = c - sk * nv;
      const int ds = sk - si + 3, dl = vl - vj + 3;
      double m = 0.0, kv = 0.0;
      if (ds >= 0 && ds < 7 && dl >= 0 && dl < 7) {
        const int sb = si * 7 + ds, vb = vj * 7 + dl;
        const double as = As[sb];
        m = as * Av[vb];
        kv = Ss[sb] * B1[vb] + Ts[sb] * B2[vb] + as * B3[vb] + St[sb] * B4[vb];
      }
      const size_t off = size_t(blk) * bs + e;
      FR[off] = FT(a_r * m + h * kv);
      if (cplx) FC[off] = cmk(FT(c_re * m + h * kv), FT(c_im * m));
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
// FP32: one reciprocal instead of two divisions (the pivot inverse is on the
// Gauss-Jordan's serial path)
__device__ __forceinline__ Cx<float> finv(Cx<float> a) {
  const float d = a.re * a.re + a.im * a.im;
  const float r = d != 0.f ? 1.f / d : 0.f;
  return cmk(a.re * r, -a.im * r);
}
__device__ __forceinline__ double fmag(float a) { return fabs(double(a)); }
__device__ __forceinline__ double fmag(double a) { return fabs(a); }
template <typename T>
__device__ __forceinline__ double fmag(Cx<T> a) {
  return sqrt(double(a.re) * double(a.re) + double(a.im) * double(a.im));
}

// --------------------------------------------------------------------------
// Stage-matrix factorization scratch (one system, ET elements).
//
// Blocks (b x b; b is called nv inside the scratch) are staged with a padded
// width nvp = b rounded up to 4 so that every tile operand is a 16-byte vector
// load and the blocks hold a whole number of register tiles (the padding is
// never written: it only meets tile rows and columns that are not stored).  GEMM left operands are stored transposed (k-major, row stride
// ldt = nvp + 4: the transposed staging writes spread over 8 banks), right
// operands row-major (stride nvp).
//   aug  nv x (nv + 1)    in-place Gauss-Jordan array of the pivot block
//   Pi   nvp x nvp        P^-1, row-major        (right operand of L = E P^-1)
//   PiT  nvp x ldt        P^-1, transposed       (left operand of W = P^-1 U)
//   EbT  bw x nvp x ldt   E_{i+1+r, i}, transposed
//   LbT  bw x nvp x ldt   L_{i+1+r, i} = E P^-1, transposed (left operand of the Schur update)
//   Ub   bw x nvp x nvp   U_{i, i+1+c}, row-major
//   pinv nvp (inverse pivot of each column), then the pivot rows prow_of and
//   their columns q_of (int)
// --------------------------------------------------------------------------
template <typename ET>
struct FacScratch {
  ET *aug, *Pi, *PiT, *EbT, *LbT, *Ub;
  ET* pinv;      // inverse pivot value of each column
  int* prow_of;  // pivot row of each column
  int* q_of;     // column whose pivot row is r
  int* claim;    // work counter of the overlapped Schur updates
  int nv, nvp, ldt, w1;
  bool shared;   // scratch in shared memory (async staging possible)
  __device__ void init(ET* base, int b, int bw) {
    nv = b;
    shared = __isShared(base) != 0;
    nvp = fpe_fac_nvp(nv);
    ldt = nvp + 4;
    w1 = nv + 1;
    const int p = nvp, t = ldt;
    aug = base;
    Pi = aug + ((nv * (nv + 1) + 3) & ~3);
    PiT = Pi + p * p;
    EbT = PiT + p * t;
    LbT = EbT + bw * p * t;
    Ub = LbT + bw * p * t;
    pinv = Ub + bw * p * p;
    prow_of = reinterpret_cast<int*>(pinv + p);
    q_of = prow_of + p;
    claim = q_of + p;
  }
};

// ---- register tiles ------------------------------------------------------
// Tile shape per element type: 4 x 4 real, 2 x 4 complex (16 FMA lanes of
// real arithmetic per operand pair either way).
template <typename ET>
struct TileM { static constexpr int v = 4; };
#ifndef FPE_CTILE_M
#define FPE_CTILE_M 2
#endif
template <typename T>
struct TileM<Cx<T>> { static constexpr int v = FPE_CTILE_M; };
// Tile width per element type (4 columns; the scratch pads blocks to a
// multiple of the widest tile).
template <typename ET>
struct TileN { static constexpr int v = 4; };

// Vector loads/stores of K consecutive elements from 16-byte aligned shared memory.
template <int K>
__device__ __forceinline__ void vld(const float* p, float (&o)[K]) {
#pragma unroll
  for (int q = 0; q < K; q += 4) {
    const float4 v = *reinterpret_cast<const float4*>(p + q);
    o[q] = v.x; o[q + 1] = v.y; o[q + 2] = v.z; o[q + 3] = v.w;
  }
}
template <int K>
__device__ __forceinline__ void vld(const double* p, double (&o)[K]) {
#pragma unroll
  for (int q = 0; q < K; q += 2) {
    const double2 v = *reinterpret_cast<const double2*>(p + q);
    o[q] = v.x; o[q + 1] = v.y;
  }
}
template <int K>
__device__ __forceinline__ void vld(const Cx<float>* p, Cx<float> (&o)[K]) {
#pragma unroll
  for (int q = 0; q < K; q += 2) {
    const float4 v = *reinterpret_cast<const float4*>(p + q);
    o[q] = cmk(v.x, v.y); o[q + 1] = cmk(v.z, v.w);
  }
}
template <int K>
__device__ __forceinline__ void vld(const Cx<double>* p, Cx<double> (&o)[K]) {
#pragma unroll
  for (int q = 0; q < K; ++q) {
    const double2 v = *reinterpret_cast<const double2*>(p + q);
    o[q] = cmk(v.x, v.y);
  }
}
template <typename ET, int K>
__device__ __forceinline__ void vst(ET* p, const ET (&v)[K]) {
#pragma unroll
  for (int q = 0; q < K; ++q) p[q] = v[q];
}

// Explicit 16-byte vector stores of a TM-element run (TM x element size is
// 16 or 32 bytes); p must be 16-byte aligned.
__device__ __forceinline__ void vst16(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void vst16(double* p, const double (&v)[4]) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void vst16(Cx<float>* p, const Cx<float> (&v)[2]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0].re, v[0].im, v[1].re, v[1].im);
}
__device__ __forceinline__ void vst16(Cx<float>* p, const Cx<float> (&v)[4]) {
  reinterpret_cast<float4*>(p)[0] = make_float4(v[0].re, v[0].im, v[1].re, v[1].im);
  reinterpret_cast<float4*>(p)[1] = make_float4(v[2].re, v[2].im, v[3].re, v[3].im);
}
__device__ __forceinline__ void vst16(Cx<double>* p, const Cx<double> (&v)[4]) {
  for (int q = 0; q < 4; ++q) reinterpret_cast<double2*>(p)[q] = make_double2(v[q].re, v[q].im);
}
__device__ __forceinline__ void vst16(Cx<double>* p, const Cx<double> (&v)[2]) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v[0].re, v[0].im);
  reinterpret_cast<double2*>(p)[1] = make_double2(v[1].re, v[1].im);
}
// K consecutive elements (K a multiple of 4) to a 16-byte aligned address.
template <typename ET, int K>
__device__ __forceinline__ void vstn(ET* p, const ET (&v)[K]) {
  static_assert(K % 4 == 0, "runs of 4 elements");
#pragma unroll
  for (int q = 0; q < K; q += 4) {
    ET w[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) w[r] = v[q + r];
    vst16(p + q, w);
  }
}

__device__ __forceinline__ void ffms(float& a, float x, float y) { a = fmaf(-x, y, a); }
__device__ __forceinline__ void ffms(double& a, double x, double y) { a = fma(-x, y, a); }
template <typename T>
__device__ __forceinline__ void ffms(Cx<T>& a, Cx<T> x, Cx<T> y) {
  a.re = fma(-x.re, y.re, a.re);
  a.re = fma(x.im, y.im, a.re);
  a.im = fma(-x.re, y.im, a.im);
  a.im = fma(-x.im, y.re, a.im);
}

// acc (+)= sum_k AT[k][j0 + m] B[k][l0 + n], k < K  (SUB: acc -= ...)
template <typename ET, bool SUB>
__device__ __forceinline__ void tile_mm(const ET* AT, int lda, const ET* B, int ldb, int K, int j0, int l0,
                                        ET (&acc)[TileM<ET>::v][TileN<ET>::v]) {
  constexpr int TM = TileM<ET>::v, kTileN = TileN<ET>::v;
  const ET* pa = AT + j0;
  const ET* pb = B + l0;
#pragma unroll 4
  for (int k = 0; k < K; ++k) {
    ET a[TM], b[kTileN];
    vld<TM>(pa + k * lda, a);
    vld<kTileN>(pb + k * ldb, b);
#pragma unroll
    for (int m = 0; m < TM; ++m)
#pragma unroll
      for (int n = 0; n < kTileN; ++n) {
        if constexpr (SUB) ffms(acc[m][n], a[m], b[n]);
        else ffma(acc[m][n], a[m], b[n]);
      }
  }
}

// ---- per block row steps ----------------------------------------------------
// Row and column of element e of an nv-wide block without an integer
// division: (e + 1/2) / nv rounded down is exact for e < 2^16.
__device__ __forceinline__ void rc_of(int e, int nv, float rnv, int& r, int& c) {
  r = int((float(e) + 0.5f) * rnv);
  c = e - r * nv;
}

// Stage block row i into the scratch: the pivot block into the Gauss-Jordan
// array, U_{i,i+1+c} row-major and E_{i+1+r,i} transposed.  With the scratch
// in shared memory the elements move by per-element asynchronous copies that
// are all in flight together; a global-memory scratch (blocks too wide for
// shared memory) is filled by ordinary loads and stores.  The caller's barrier
// follows.
template <typename ET, bool ASYNC>
__device__ __forceinline__ void stage_elem(ET* dst, const ET* src) {
  if constexpr (ASYNC) {
    cp_async_elem<int(sizeof(ET))>(dst, src);
  } else {
    *dst = *src;
  }
}

// Stages block row i: with PIVOT its pivot block (into the Gauss-Jordan
// array, and the pivot bookkeeping reset), with REST the nr U blocks of row i
// and E blocks of column i.
template <typename ET, bool ASYNC>
__device__ __forceinline__ void fac_stage_impl(const BlockLU<ET>& L, FacScratch<ET>& S, int i, int nr, bool pivot, bool rest) {
  const int nv = S.nv, nn = nv * nv, w1 = S.w1, p = S.nvp, t = S.ldt;
  const float rnv = 1.0f / float(nv);
  if (pivot) {
    const ET* P = L.blk(i, L.bw);
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
      int r, c;
      rc_of(e, nv, rnv, r, c);
      stage_elem<ET, ASYNC>(S.aug + r * w1 + c, P + e);
    }
    for (int r = threadIdx.x; r < nv; r += blockDim.x) {
      S.q_of[r] = r;  // stays a valid column index even if a pivot search fails
      S.prow_of[r] = r;
    }
  }
  if (rest) {
    for (int cc = 0; cc < nr; ++cc) {
      const ET* U = L.blk(i, L.bw + 1 + cc);
      const ET* E = L.blk(i + 1 + cc, L.bw - 1 - cc);
      ET* ub = S.Ub + cc * p * p;
      ET* et = S.EbT + cc * p * t;
      for (int e = threadIdx.x; e < nn; e += blockDim.x) {
        int j, l;
        rc_of(e, nv, rnv, j, l);
        stage_elem<ET, ASYNC>(ub + j * p + l, U + e);
        stage_elem<ET, ASYNC>(et + l * t + j, E + e);
      }
    }
  }
  if constexpr (ASYNC) cp_async_wait_all();
}

template <typename ET>
__device__ __forceinline__ void fac_stage(const BlockLU<ET>& L, FacScratch<ET>& S, int i, int nr, bool pivot = true,
                          bool rest = true) {
  if (S.shared) {
    fac_stage_impl<ET, true>(L, S, i, nr, pivot, rest);
  } else {
    fac_stage_impl<ET, false>(L, S, i, nr, pivot, rest);
  }
}

// |re| + |im| (LAPACK's cabs1) as the pivot magnitude, in float.
__device__ __forceinline__ float pmag(float a) { return fabsf(a); }
__device__ __forceinline__ float pmag(double a) { return float(fabs(a)); }
template <typename T>
__device__ __forceinline__ float pmag(Cx<T> a) {
  return float(fabs(double(a.re)) + fabs(double(a.im)));
}
__device__ __forceinline__ float pmag(Cx<float> a) { return fabsf(a.re) + fabsf(a.im); }

// Pivot key of row r: the magnitude's float bits above bit 7, then 127 - r,
// so one unsigned max over the warp picks the largest magnitude and, among
// equal keys, the lowest row.  Rows already pivotal have key 0.
__device__ __forceinline__ unsigned pivot_key(float m, int r) {
  return (__float_as_uint(m) & ~127u) | unsigned(127 - r);
}

template <typename ET>
struct IsF32Elem { static constexpr bool v = false; };
template <>
struct IsF32Elem<float> { static constexpr bool v = true; };
template <>
struct IsF32Elem<Cx<float>> { static constexpr bool v = true; };

// One Gauss-Jordan update a - f p: fused multiply-adds for FP32 elements
// (fewer instructions on the inversion's serial path), a rounded product then
// a difference for FP64 ones.
template <typename ET>
__device__ __forceinline__ ET gj_elim(ET a, ET f, ET p) {
  if constexpr (IsF32Elem<ET>::v) {
    ffms(a, f, p);
    return a;
  } else {
    return fsub(a, fmul(f, p));
  }
}

// In-place Gauss-Jordan inversion of the staged pivot block by one warp, with
// unscaled pivot rows:  for column c with pivot row p and f_r = a_rc / a_pc,
//   a_rl -= f_r a_pl (r != p, all l),   a_rc = -f_r (r != p),   a_pc = 1.
// Lane r owns rows r and r + 32, so a step touches only the lane's own rows
// and reads the pivot row, which no lane writes during that step.  After the
// last column, row p_k divided by the pivot a_{p_k k} holds row k of P^-1 with
// its columns in pivot order (column q_l holds inverse column l).  Returns
// false for a zero or non-finite pivot.
template <typename ET>
__device__ __forceinline__ bool fac_gj_warp(FacScratch<ET>& S) {
  const int lane = threadIdx.x & 31, nv = S.nv, w1 = S.w1;
  const int r0 = lane, r1 = lane + 32;
  const bool own0 = r0 < nv, own1 = r1 < nv;
  bool used0 = false, used1 = false, ok = true;
  ET* a0 = S.aug + r0 * w1;
  ET* a1 = S.aug + r1 * w1;
  for (int c = 0; c < nv; ++c) {
    unsigned k = 0;
    if (own0 && !used0) k = pivot_key(pmag(a0[c]), r0);
    if (own1 && !used1) k = max(k, pivot_key(pmag(a1[c]), r1));
    const unsigned kmax = __reduce_max_sync(0xffffffffu, k);
    const int p = min(127 - int(kmax & 127u), nv - 1);  // an unused row always has a nonzero key
    const ET* ap = S.aug + p * w1;
    const ET pv = ap[c];
    const float pm = pmag(pv);
    ok &= (pm > 0.f) && (pm < CUDART_INF_F);
    const ET inv = finv(pv);
    if (p == r0) used0 = true;
    if (p == r1) used1 = true;
    if (lane == 0) {
      S.prow_of[c] = p;
      S.q_of[p] = c;
      S.pinv[c] = inv;
    }
    __syncwarp();  // every lane has read a_pc before the owner overwrites it
    // row -= f * pivot row, in 8-element chunks loaded to registers before any
    // store (the rows never alias, but the compiler cannot know), so the
    // shared-memory loads of a chunk overlap instead of forming one chain
    auto eliminate = [&](ET* row) {
      const ET f = fmul(row[c], inv);
      int l = 0;
      for (; l + 8 <= nv; l += 8) {
        ET pv[8], rv[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          pv[k] = ap[l + k];
          rv[k] = row[l + k];
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) row[l + k] = gj_elim(rv[k], f, pv[k]);
      }
      for (; l < nv; ++l) row[l] = gj_elim(row[l], f, ap[l]);
      row[c] = fsub(fzero(ET()), f);
    };
    if (own0 && r0 != p) eliminate(a0);
    if (own1 && r1 != p) eliminate(a1);
    if (p == r0) a0[c] = fone(ET());
    if (p == r1) a1[c] = fone(ET());
    __syncwarp();
  }
  return ok;
}

// Lane-to-lane copy of a register element (the pivot row's broadcast).
__device__ __forceinline__ float shfl_elem(float v, int src) { return __shfl_sync(0xffffffffu, v, src); }
__device__ __forceinline__ Cx<float> shfl_elem(Cx<float> v, int src) {
  return cmk(__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src));
}

// The same Gauss-Jordan inversion with each lane's row in registers (FP32
// blocks of NV <= 32 columns): lane r keeps row r for the whole inversion,
// and each step broadcasts the pivot row from its lane by shuffles (no
// shared-memory round trip, no divergent stores).  The row rotates left by
// four columns every four steps, so the current column is one of elements
// 0..3 and the loop body is four compiled steps (register indices are
// compile-time); after NV steps the columns are back in order.  The pivot
// choice, the arithmetic of each element and the bookkeeping are those of
// fac_gj_warp.
template <typename ET, int NV>
__device__ __noinline__ bool fac_gj_warp_reg(uint32_t aug_off, uint32_t pinv_off, uint32_t prow_off,
                                              uint32_t qof_off) {
  static_assert(NV <= 32 && NV % 4 == 0, "register rows of up to 32 columns, 16-byte chunks");
  // the scratch arrays, rebuilt from shared offsets so that their accesses are LDS / STS
  ET* const aug = reinterpret_cast<ET*>(fpe_dsmem + aug_off);
  ET* const pinv = reinterpret_cast<ET*>(fpe_dsmem + pinv_off);
  int* const prow_of = reinterpret_cast<int*>(fpe_dsmem + prow_off);
  int* const q_of = reinterpret_cast<int*>(fpe_dsmem + qof_off);
  const int lane = threadIdx.x & 31, w1 = NV + 1;
  const bool own = lane < NV;
  ET row[NV];
#pragma unroll
  for (int l = 0; l < NV; ++l) row[l] = own ? aug[lane * w1 + l] : fzero(ET());
  bool used = false, ok = true;
#pragma unroll 1
  for (int c0 = 0; c0 < NV; c0 += 4) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int c = c0 + u;
      const unsigned k = (own && !used) ? pivot_key(pmag(row[u]), lane) : 0u;
      const unsigned kmax = __reduce_max_sync(0xffffffffu, k);
      const int p = min(127 - int(kmax & 127u), NV - 1);  // an unused row always has a nonzero key
      const ET pv = shfl_elem(row[u], p);
      ET q[NV];
#pragma unroll
      for (int l = 0; l < NV; ++l) q[l] = l == u ? pv : shfl_elem(row[l], p);
      const float pm = pmag(pv);
      ok &= (pm > 0.f) && (pm < CUDART_INF_F);
      const ET inv = finv(pv);
      if (lane == 0) {
        prow_of[c] = p;
        q_of[p] = c;
        pinv[c] = inv;
      }
      if (lane == p) {
        used = true;
        row[u] = fone(ET());
      } else if (own) {
        const ET f = fmul(row[u], inv);
#pragma unroll
        for (int l = 0; l < NV; ++l)
          if (l != u) row[l] = gj_elim(row[l], f, q[l]);
        row[u] = fsub(fzero(ET()), f);
      }
    }
    ET t[4];
#pragma unroll
    for (int l = 0; l < 4; ++l) t[l] = row[l];
#pragma unroll
    for (int l = 0; l + 4 < NV; ++l) row[l] = row[l + 4];
#pragma unroll
    for (int l = 0; l < 4; ++l) row[NV - 4 + l] = t[l];
  }
  if (own) {
#pragma unroll
    for (int l = 0; l < NV; ++l) aug[lane * w1 + l] = row[l];
  }
  return ok;
}

// The pivot-block inverse: rows in registers for FP32 blocks of 8 to 32
// columns (multiples of 4), rows in shared memory otherwise.
template <typename ET>
__device__ __forceinline__ bool fac_gj(FacScratch<ET>& S) {
  if constexpr (IsF32Elem<ET>::v) {
    if (S.shared) {
      const uint32_t a = dsmem_offset(S.aug), pi = dsmem_offset(S.pinv), pr = dsmem_offset(S.prow_of),
                     qo = dsmem_offset(S.q_of);
      switch (S.nv) {
        case 8: return fac_gj_warp_reg<ET, 8>(a, pi, pr, qo);
        case 12: return fac_gj_warp_reg<ET, 12>(a, pi, pr, qo);
        case 16: return fac_gj_warp_reg<ET, 16>(a, pi, pr, qo);
        case 24: return fac_gj_warp_reg<ET, 24>(a, pi, pr, qo);
        case 32: return fac_gj_warp_reg<ET, 32>(a, pi, pr, qo);
        default: break;
      }
    }
  }
  return fac_gj_warp<ET>(S);
}

// P^-1 (row k = row p_k of the array scaled by 1 / a_{p_k k}, columns
// un-permuted) into Pi, PiT and the factor storage.
template <typename ET>
__device__ __forceinline__ void fac_extract(const BlockLU<ET>& L, FacScratch<ET>& S, int i) {
  const int nv = S.nv, w1 = S.w1, p = S.nvp, t = S.ldt;
  const float rnv = 1.0f / float(nv);
  ET* g = L.blk(i, L.bw);
  // k varying fastest: the transposed factor store and PiT are contiguous
  for (int e = threadIdx.x; e < nv * nv; e += blockDim.x) {
    int l, k;
    rc_of(e, nv, rnv, l, k);
    const ET v = fmul(S.aug[S.prow_of[k] * w1 + S.q_of[l]], S.pinv[k]);
    S.PiT[l * t + k] = v;
    g[e] = v;  // stored transposed: g[l nv + k]
  }
  // l varying fastest: Pi is contiguous
  for (int e = threadIdx.x; e < nv * nv; e += blockDim.x) {
    int k, l;
    rc_of(e, nv, rnv, k, l);
    S.Pi[k * p + l] = fmul(S.aug[S.prow_of[k] * w1 + S.q_of[l]], S.pinv[k]);
  }
}

// L_r = E_r P^-1 (transposed to the factor storage and to LbT) and
// W_c = P^-1 U_c (transposed to the factor storage), r, c < nr.  Tiles are
// numbered with the row index j varying fastest, so that a lane's TM rows of
// one output column are contiguous in the transposed storage: one vector
// store each, and a warp's stores cover contiguous memory.
// Tile tt of job `job` (job < nr: L_job; else W_{job - nr}).
template <typename ET>
__device__ __forceinline__ void fac_lw_tile(const BlockLU<ET>& L, FacScratch<ET>& S, int i, int nr, int job, int tt) {
  constexpr int TM = TileM<ET>::v, kTileN = TileN<ET>::v;
  const int nv = S.nv, p = S.nvp, t = S.ldt;
  const int tr = p / TM;
  const bool vec = ((nv * int(sizeof(ET))) & 15) == 0 && ((L.bs * sizeof(ET)) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(L.F) & 15) == 0;
  const int l0 = (tt / tr) * kTileN, j0 = (tt - (tt / tr) * tr) * TM;
  ET acc[TM][kTileN];
#pragma unroll
  for (int m = 0; m < TM; ++m)
#pragma unroll
    for (int n = 0; n < kTileN; ++n) acc[m][n] = fzero(ET());
  ET* dst;
  if (job < nr) {
    tile_mm<ET, false>(S.EbT + job * p * t, t, S.Pi, p, nv, j0, l0, acc);
    dst = L.blk(i + 1 + job, L.bw - 1 - job);
    ET* lt = S.LbT + job * p * t;
#pragma unroll
    for (int n = 0; n < kTileN; ++n) {
      ET col[TM];
#pragma unroll
      for (int m = 0; m < TM; ++m) col[m] = acc[m][n];
      vst<ET, TM>(lt + (l0 + n) * t + j0, col);
    }
  } else {
    const int cc = job - nr;
    tile_mm<ET, false>(S.PiT, t, S.Ub + cc * p * p, p, nv, j0, l0, acc);
    dst = L.blk(i, L.bw + 1 + cc);
  }
  if (vec && j0 + TM <= nv) {
#pragma unroll
    for (int n = 0; n < kTileN; ++n) {
      if (l0 + n < nv) {
        ET col[TM];
#pragma unroll
        for (int m = 0; m < TM; ++m) col[m] = acc[m][n];
        vst16(dst + (l0 + n) * nv + j0, col);
      }
    }
  } else {
#pragma unroll
    for (int m = 0; m < TM; ++m)
#pragma unroll
      for (int n = 0; n < kTileN; ++n)
        if (j0 + m < nv && l0 + n < nv) dst[(l0 + n) * nv + j0 + m] = acc[m][n];
  }
}

template <typename ET>
__device__ __forceinline__ void fac_lw(const BlockLU<ET>& L, FacScratch<ET>& S, int i, int nr) {
  const int ntile = (S.nvp / TileM<ET>::v) * (S.nvp / TileN<ET>::v);
  for (int q = threadIdx.x; q < 2 * nr * ntile; q += blockDim.x) {
    const int job = q / ntile;
    fac_lw_tile<ET>(L, S, i, nr, job, q - job * ntile);
  }
}

// Schur update E_{i+1+r, i+1+c} -= L_r U_c (r, c < nr) for the jobs
// job_lo <= r nr + c < job_hi, by threads lt = 0 .. nt - 1 of a team; the
// target tile is loaded first so its latency overlaps the products.  Job 0
// (the next pivot block E_{i+1, i+1}) goes with TO_AUG into the Gauss-Jordan
// array instead of the factor storage: the next block row inverts it from
// there, and the factor storage of that block receives its inverse.
template <typename ET>
__device__ __forceinline__ int fac_tiles(const FacScratch<ET>& S) {
  return (S.nvp / TileM<ET>::v) * (S.nvp / TileN<ET>::v);
}

// Tile q of the Schur jobs job_lo, job_lo + 1, ... (q = job offset x tiles per
// job + tile).
template <typename ET, bool TO_AUG>
__device__ __forceinline__ void fac_update_tile(const BlockLU<ET>& L, FacScratch<ET>& S, int i, int nr, int job_lo,
                                                int q) {
  constexpr int TM = TileM<ET>::v, kTileN = TileN<ET>::v;
  const int nv = S.nv, p = S.nvp, t = S.ldt;
  const int tc = p / kTileN, ntile = fac_tiles(S);
  {
    const int jq = q / ntile, tt = q - jq * ntile, job = job_lo + jq;
    const int j0 = (tt / tc) * TM, l0 = (tt - (tt / tc) * tc) * kTileN;
    const int rr = job / nr, cc = job - rr * nr;
    ET* E = L.blk(i + 1 + rr, cc - rr + L.bw);
    ET acc[TM][kTileN];
    if constexpr (IsF32Elem<ET>::v) {
      // FP32: the products accumulate from zero and the target tile (global
      // memory, written by the previous block row's updates) is subtracted
      // at the end, so its loads are in flight while the products run
      // instead of holding up the first one
      ET e[TM][kTileN];
      const bool vec = (nv & 3) == 0 && l0 + kTileN <= nv;  // rows of the tile are 16-byte aligned runs
#pragma unroll
      for (int m = 0; m < TM; ++m) {
        if (vec && j0 + m < nv) {
          vld<kTileN>(E + (j0 + m) * nv + l0, e[m]);
        } else {
#pragma unroll
          for (int n = 0; n < kTileN; ++n)
            e[m][n] = (j0 + m < nv && l0 + n < nv) ? E[(j0 + m) * nv + l0 + n] : fzero(ET());
        }
#pragma unroll
        for (int n = 0; n < kTileN; ++n) acc[m][n] = fzero(ET());
      }
      tile_mm<ET, false>(S.LbT + rr * p * t, t, S.Ub + cc * p * p, p, nv, j0, l0, acc);
#pragma unroll
      for (int m = 0; m < TM; ++m)
#pragma unroll
        for (int n = 0; n < kTileN; ++n) acc[m][n] = fsub(e[m][n], acc[m][n]);
    } else {
#pragma unroll
      for (int m = 0; m < TM; ++m)
#pragma unroll
        for (int n = 0; n < kTileN; ++n)
          acc[m][n] = (j0 + m < nv && l0 + n < nv) ? E[(j0 + m) * nv + l0 + n] : fzero(ET());
      tile_mm<ET, true>(S.LbT + rr * p * t, t, S.Ub + cc * p * p, p, nv, j0, l0, acc);
    }
    if constexpr (TO_AUG) {
#pragma unroll
      for (int m = 0; m < TM; ++m)
#pragma unroll
        for (int n = 0; n < kTileN; ++n)
          if (j0 + m < nv && l0 + n < nv) S.aug[(j0 + m) * S.w1 + l0 + n] = acc[m][n];
    } else if ((nv & 3) == 0 && l0 + kTileN <= nv) {
#pragma unroll
      for (int m = 0; m < TM; ++m)
        if (j0 + m < nv) vstn(E + (j0 + m) * nv + l0, acc[m]);
    } else {
#pragma unroll
      for (int m = 0; m < TM; ++m)
#pragma unroll
        for (int n = 0; n < kTileN; ++n)
          if (j0 + m < nv && l0 + n < nv) E[(j0 + m) * nv + l0 + n] = acc[m][n];
    }
  }
}

template <typename ET, bool TO_AUG>
__device__ __forceinline__ void fac_update(const BlockLU<ET>& L, FacScratch<ET>& S, int i, int nr, int job_lo, int job_hi, int lt,
                           int nt) {
  for (int q = lt; q < (job_hi - job_lo) * fac_tiles(S); q += nt) fac_update_tile<ET, TO_AUG>(L, S, i, nr, job_lo, q);
}

// Schur updates 1 .. nr^2 - 1 of both systems, claimed 32 tiles at a time
// per warp, so that the warps which finish their pivot inverse early take
// their share of the products: the complex tiles first (counter ctr[0]), then
// the real ones (ctr[1], four times less work a tile, which evens out the
// warps' finishing times).  One loop per element type keeps each loop's
// registers to one tile shape.
template <typename FT>
__device__ __forceinline__ void fac_update_claim(const BlockLU<FT>& LR, FacScratch<FT>& SR, const BlockLU<Cx<FT>>* LC,
                                 FacScratch<Cx<FT>>& SC, int i, int nr, int* ctr) {
  const int lane = threadIdx.x & 31;
  if (LC) {
    const int total = (nr * nr - 1) * fac_tiles(SC);
    for (;;) {
      int base = 0;
      if (lane == 0) base = atomicAdd(ctr, 32);
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= total) break;
      if (base + lane < total) fac_update_tile<Cx<FT>, false>(*LC, SC, i, nr, 1, base + lane);
    }
  }
  const int total = (nr * nr - 1) * fac_tiles(SR);
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(ctr + 1, 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= total) break;
    if (base + lane < total) fac_update_tile<FT, false>(LR, SR, i, nr, 1, base + lane);
  }
}

// Factor the real stage matrix (and, when LC is given, the complex one in
// lockstep so both share every barrier).  scr_r / scr_c: scratch of
// fpe_fac_scratch_elems(b, bw) elements each.
template <typename FT>
__device__ __forceinline__ bool blu_factor_pair(const BlockLU<FT>& LR, const BlockLU<Cx<FT>>* LC, FT* scr_r,
                                Cx<FT>* scr_c, long long (&tcyc)[4]) {
  const int ns = LR.nb, bw = LR.bw;  // block rows, off-diagonal blocks
  long long tc0 = 0, tc1 = 0, tc2 = 0, tc3 = 0;  // phase timers in registers, added to tcyc at the end
  FacScratch<FT> SR;
  SR.init(scr_r, LR.b, bw);
  FacScratch<Cx<FT>> SC;
  if (LC) SC.init(scr_c, LR.b, bw);
  bool ok = true;
  const int warp = threadIdx.x >> 5;
  // Lookahead: block row i computes the next pivot block first (Schur job 0,
  // straight into the Gauss-Jordan array); warps 0 and 1 then invert it (real,
  // complex) while warps 2.. apply row i's remaining Schur updates, so the
  // latency-bound inversions overlap the block products.  Block row 0 stages
  // and inverts its own pivot block.
  const bool split = blockDim.x >= 128;
  if (ns <= 0) return true;
  {
    const long long t0 = clock64();
    fac_stage<FT>(LR, SR, 0, min(bw, ns - 1));
    if (LC) fac_stage<Cx<FT>>(*LC, SC, 0, min(bw, ns - 1));
    __syncthreads();
    if (warp == 0) ok &= FPE_GJ<FT>(SR);
    else if (warp == 1 && LC) ok &= FPE_GJ<Cx<FT>>(SC);
    __syncthreads();
    tc0 += clock64() - t0;
  }
  for (int i = 0; i < ns; ++i) {
    const int nr = min(i + bw, ns - 1) - i;
    const long long t1 = clock64();
    if (i > 0) {  // U and E blocks of row i (its pivot block is already inverted)
      fac_stage<FT>(LR, SR, i, nr, false, true);
      if (LC) fac_stage<Cx<FT>>(*LC, SC, i, nr, false, true);
      __syncthreads();
    }
    fac_extract<FT>(LR, SR, i);
    if (LC) fac_extract<Cx<FT>>(*LC, SC, i);
    __syncthreads();
    tc3 += clock64() - t1;
    if (nr > 0) {
      const long long t2 = clock64();
      fac_lw<FT>(LR, SR, i, nr);
      if (LC) fac_lw<Cx<FT>>(*LC, SC, i, nr);
      __syncthreads();
      // the next pivot block into the Gauss-Jordan arrays; fresh bookkeeping
      fac_update<FT, true>(LR, SR, i, nr, 0, 1, threadIdx.x, blockDim.x);
      if (LC) fac_update<Cx<FT>, true>(*LC, SC, i, nr, 0, 1, threadIdx.x, blockDim.x);
      for (int r = threadIdx.x; r < SR.nv; r += blockDim.x) {
        SR.q_of[r] = r;
        SR.prow_of[r] = r;
        if (LC) {
          SC.q_of[r] = r;
          SC.prow_of[r] = r;
        }
      }
      if (threadIdx.x == 0) {
        SR.claim[0] = 0;
        SR.claim[1] = 0;
      }
      __syncthreads();
      const long long t3 = clock64();
      tc1 += t3 - t2;
      if (split) {
        if (warp == 0) {
          ok &= FPE_GJ<FT>(SR);
        } else if (warp == 1) {
          if (LC) ok &= FPE_GJ<Cx<FT>>(SC);
        }
        fac_update_claim<FT>(LR, SR, LC, SC, i, nr, SR.claim);
        // this warp's own time in the overlapped phase, before the barrier
        tc2 += clock64() - t3;
      } else {
        fac_update<FT, false>(LR, SR, i, nr, 1, nr * nr, threadIdx.x, blockDim.x);
        if (LC) fac_update<Cx<FT>, false>(*LC, SC, i, nr, 1, nr * nr, threadIdx.x, blockDim.x);
        __syncthreads();
        if (warp == 0) ok &= FPE_GJ<FT>(SR);
        else if (warp == 1 && LC) ok &= FPE_GJ<Cx<FT>>(SC);
      }
      __syncthreads();
      tc0 += clock64() - t3;
    }
  }
  tcyc[0] += tc0;
  tcyc[1] += tc1;
  tcyc[2] += tc2;
  tcyc[3] += tc3;
  return __syncthreads_and(ok ? 1 : 0) != 0;  // the same verdict in every thread
}

// The factorization with its scratch in shared memory, compiled as a
// function of its own: it gets a register allocation of its own (the kernel
// around it is large), its block descriptions arrive by value, and its
// scratch as shared-window offsets, so that no read in its loops goes to the
// kernel's stack frame and every scratch access is a shared-memory
// instruction.  tcyc accumulates the phase timers of blu_factor_pair.
template <typename FT>
__device__ __noinline__ bool blu_factor_pair_smem(BlockLU<FT> LR, BlockLU<Cx<FT>> LC, bool cplx, uint32_t scr_r,
                                                  uint32_t scr_c, long long* tcyc) {
  long long tc[4] = {0, 0, 0, 0};
  const bool ok = blu_factor_pair<FT>(LR, cplx ? &LC : nullptr, reinterpret_cast<FT*>(fpe_dsmem + scr_r),
                                      reinterpret_cast<Cx<FT>*>(fpe_dsmem + scr_c), tc);
#pragma unroll
  for (int k = 0; k < 4; ++k) tcyc[k] += tc[k];
  return ok;
}

// The same with the scratch in global memory (blocks too wide for shared
// memory), also out of line.
template <typename FT>
__device__ __noinline__ bool blu_factor_pair_gmem(BlockLU<FT> LR, BlockLU<Cx<FT>> LC, bool cplx, FT* scr_r,
                                                  Cx<FT>* scr_c, long long* tcyc) {
  long long tc[4] = {0, 0, 0, 0};
  const bool ok = blu_factor_pair<FT>(LR, cplx ? &LC : nullptr, scr_r, scr_c, tc);
#pragma unroll
  for (int k = 0; k < 4; ++k) tcyc[k] += tc[k];
  return ok;
}

// Right-hand sides of one fused solve: up to two real vectors on the real
// factor and one complex vector (re, im arrays) on the complex factor.  The
// factors' descriptions are held by value (both share their block structure;
// R's describes it); the staged solve reads the members it needs into scalars
// once per sweep.
template <typename FT>
struct SolveSet {
  BlockLU<FT> R;
  BlockLU<Cx<FT>> Cf;
  double* xr[2];   // in: b, out: x
  double* zr[2];   // scratch N
  int nr;
  double* xc_re;
  double* xc_im;
  double* zc_re;
  double* zc_im;
  int nc;  // 0 or 1
};

// Dot product of row j of a stored (transposed) factor block with x over the
// lanes gl, gl + G, ... of a group: col = block + j, element m at col[m nv].
template <typename ET, typename A>
__device__ __forceinline__ A grp_dot(const ET* col, const double* xre, const double* xim, int nv, int gl, int G);

template <>
__device__ __forceinline__ double grp_dot<float, double>(const float* col, const double* x, const double*, int nv,
                                                         int gl, int G) {
  double a = 0.0;
  for (int m = gl; m < nv; m += G) a = fma(double(col[m * nv]), x[m], a);
  return a;
}
template <>
__device__ __forceinline__ double grp_dot<double, double>(const double* col, const double* x, const double*,
                                                          int nv, int gl, int G) {
  double a = 0.0;
  for (int m = gl; m < nv; m += G) a = fma(col[m * nv], x[m], a);
  return a;
}
template <>
__device__ __forceinline__ Cx<double> grp_dot<Cx<float>, Cx<double>>(const Cx<float>* col, const double* xr,
                                                                      const double* xi, int nv, int gl, int G) {
  Cx<double> a = cmk(0.0, 0.0);
  for (int m = gl; m < nv; m += G) afma(a, acc_load(col[m * nv]), cmk(xr[m], xi[m]));
  return a;
}
template <>
__device__ __forceinline__ Cx<double> grp_dot<Cx<double>, Cx<double>>(const Cx<double>* col, const double* xr,
                                                                       const double* xi, int nv, int gl, int G) {
  Cx<double> a = cmk(0.0, 0.0);
  for (int m = gl; m < nv; m += G) afma(a, col[m * nv], cmk(xr[m], xi[m]));
  return a;
}

// Fused block solve of all right-hand sides in S (2 ns + 1 barriers).  Thread
// groups of G lanes own one row of one system; every lane executes the same
// shuffle reductions (real systems carry a zero imaginary part).
template <typename FT>
__device__ __forceinline__ void blu_solve(const SolveSet<FT>& Sin) {
  const SolveSet<FT> S = Sin;  // in registers for the sweep
  const int ns = S.R.nb;   // block rows
  const int nv = S.R.b;    // block size
  const int bw = S.R.bw;
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
      const BlockLU<FT>& L = S.R;
      const double* x = S.xr[sys];
      if (i < ns)
        for (int k = 1; k <= bw && i - k >= 0; ++k)
          ar += grp_dot<FT, double>(L.blk(i, bw - k) + j, x + (i - k) * nv, nullptr, nv, gl, G);
      if (i > 0) zr = grp_dot<FT, double>(L.blk(i - 1, bw) + j, x + (i - 1) * nv, nullptr, nv, gl, G);
    } else if (is_c) {
      const BlockLU<Cx<FT>>& L = S.Cf;
      if (i < ns)
        for (int k = 1; k <= bw && i - k >= 0; ++k) {
          const Cx<double> d = grp_dot<Cx<FT>, Cx<double>>(L.blk(i, bw - k) + j, S.xc_re + (i - k) * nv,
                                                           S.xc_im + (i - k) * nv, nv, gl, G);
          ar += d.re;
          ai += d.im;
        }
      if (i > 0) {
        const Cx<double> d = grp_dot<Cx<FT>, Cx<double>>(L.blk(i - 1, bw) + j, S.xc_re + (i - 1) * nv,
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
      const BlockLU<FT>& L = S.R;
      const double* x = S.xr[sys];
      for (int k = 1; k <= bw && i + k < ns; ++k)
        ar += grp_dot<FT, double>(L.blk(i, bw + k) + j, x + (i + k) * nv, nullptr, nv, gl, G);
    } else if (is_c) {
      const BlockLU<Cx<FT>>& L = S.Cf;
      for (int k = 1; k <= bw && i + k < ns; ++k) {
        const Cx<double> d = grp_dot<Cx<FT>, Cx<double>>(L.blk(i, bw + k) + j, S.xc_re + (i + k) * nv,
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


// --------------------------------------------------------------------------
// Staged fused block solve.
//
// The 2 nb + 1 block rows of a solve (forward rows 0..nb, backward rows
// nb-1..0) stream through nbuf (2 to 4) shared-memory stage buffers by bulk
// copies: while the CTA multiplies stage s, stages s + 1 .. s + nbuf - 1 are
// in flight, and one thread issues stage s + nbuf into the freed buffer after
// the row's barrier, so each copy has nbuf - 1 stage times to land.  A stage
// holds the blocks the row needs from each factor (forward row i:
// L_{i,i-bw+g}, g < bw, and P^-1_{i-1}; backward row i: W_{i,i+1+g}), one slot
// per block with a 64-byte gap so that the slots of a complex row group start
// in alternate bank halves.  The last bw + 1 solved block segments of every
// right-hand side stay in a shared ring (a power of two of segments), so each
// row reads its x operands from shared memory.
// One thread owns one row of a real system; Gc lanes own one row of the
// complex system and split its blocks.
// --------------------------------------------------------------------------
constexpr int kMaxStageBufs = 4;

struct SolveStage {
  unsigned char* buf[kMaxStageBufs];  // stage buffers (shared, 16-byte aligned)
  int nbuf;                  // buffers in use (2 .. kMaxStageBufs)
  void* ring;                // ring_segments(bw) segments x b per right-hand-side array (nr real,
                             // re, im), of the sweep's accumulation type (float with FP32
                             // factors, else double)
  unsigned long long* bar;   // nbuf mbarriers (shared)
  int* err;                  // shared flag: a bounded wait gave up
  int slot_r, slot_c;        // bytes per staged real / complex block slot
  long long wait_limit;      // SM cycles a stage waits for its copies
  long long* wait_cycles;    // accumulates this thread's cycles spent in those waits
  long long* work_cycles;    // ... in a stage's work after the wait
  long long* bar_cycles;     // ... at the stage barriers
  bool rhs_bulk;             // forward stages bring their right-hand-side segments along
                             // (block size even: 16-byte aligned segments)
  void* zbuf;                // shared z = P^-1 y of the forward sweep (null: global scratch)
  int zcap;                  // bytes of zbuf
};

__host__ __device__ __forceinline__ int stage_slot_bytes(int b, int esz) {
  return fpe_block_stride(b) * esz + 64;
}
// Segments of the sweep's ring: bw + 1 rounded up to a power of two.
__host__ __device__ __forceinline__ int ring_segments(int bw) { return bw < 4 ? 4 : 8; }
// Bytes of one stage buffer for block size b, element size esz of the real
// factor, with or without the complex factor: bw + 1 factor-block slots, then
// up to four right-hand-side segments of b doubles (offset stage_rhs_offset).
__host__ __device__ __forceinline__ int stage_rhs_offset(int b, int esz, bool cplx, int bw) {
  return (bw + 1) * (stage_slot_bytes(b, esz) + (cplx ? stage_slot_bytes(b, 2 * esz) : 0));
}
__host__ __device__ __forceinline__ int stage_bytes(int b, int esz, bool cplx, int bw) {
  return stage_rhs_offset(b, esz, cplx, bw) + ((4 * b * 8 + 15) & ~15);
}
// Bytes of nbuf stage buffers plus the ring (up to 4 arrays of 8-byte entries).
__host__ __device__ __forceinline__ int stage_total_bytes(int b, int esz, bool cplx, int bw, int nbuf) {
  return nbuf * stage_bytes(b, esz, cplx, bw) + ring_segments(bw) * b * 4 * 8;
}

// The copies of a sweep's stages as the issuing thread sees them: factor
// bases, shared-window addresses of the stage buffers and their barriers, and
// the right-hand sides, all scalars.  No member is an array, so nothing is
// indexed at run time and the whole description stays in registers (a
// run-time index into a struct array places it in local memory, whose loads
// miss the small L1 left beside a large shared-memory carve-out and would put
// hundreds of cycles on every stage).
template <typename FT, int BW>
struct StageCopies {
  const unsigned char* fr;  // real factor (bytes); null: no real system
  const unsigned char* fc;  // complex factor (bytes); null: no complex system
  uint32_t br;              // bytes per real block (a complex block is 2 br)
  int nb;                   // block rows
  uint32_t dst0, dstep;     // shared address of stage buffer 0, bytes between buffers
  uint32_t slot_r, slot_c;  // bytes per staged real / complex block slot
  uint32_t rhs_at;          // offset of the right-hand-side segments in a buffer
  uint32_t bar0;            // shared address of barrier 0 (8 bytes per barrier)
  uint32_t seg;             // bytes of one right-hand-side segment (b doubles)
  const double *x0, *x1, *xre, *xim;  // right-hand sides (null: none)
  bool rhs;                 // forward stages bring their right-hand-side segments

  // Block kk of factor row i as a byte offset from the factor base.
  __device__ __forceinline__ size_t boff(int i, int kk, uint32_t bb) const {
    return (size_t(i) * (2 * BW + 1) + kk) * bb;
  }
  // Slot g of stage s: whether the row has the block, and its (row, column
  // slot).  Forward row i = s <= nb: L_{i,i-BW+g} for g < BW, P^-1_{i-1} for
  // g = BW; backward row i = 2 nb - s: W_{i,i+1+g} for g < BW.
  __device__ __forceinline__ bool slot(int s, int g, int& i, int& kk) const {
    if (s <= nb) {
      if (g < BW) {
        i = s;
        kk = g;
        return s < nb && s - BW + g >= 0;
      }
      i = s - 1;
      kk = BW;
      return s >= 1;
    }
    i = 2 * nb - s;
    kk = BW + 1 + g;
    return g < BW && i + 1 + g < nb;
  }
  // Issues the copies of stage s into buffer b.  gfence orders the factor's
  // earlier generic-proxy writes (the factorization) before the async-proxy
  // reads; the factor does not change during a sweep, so only a sweep's first
  // issue needs it.
  __device__ __forceinline__ void issue(int s, int b, bool gfence) const {
    constexpr int ng = BW + 1;
    const uint32_t bar = bar0 + 8u * uint32_t(b);
    const uint32_t dst = dst0 + uint32_t(b) * dstep;
    const bool rrow = rhs && s < nb;  // forward rows 0 .. nb-1 read b_s
    int nblk = 0;
#pragma unroll
    for (int g = 0; g < ng; ++g) {
      int i, kk;
      nblk += slot(s, g, i, kk) ? 1 : 0;
    }
    const int nrhs = rrow ? (x0 ? 1 : 0) + (x1 ? 1 : 0) + (xre ? 2 : 0) : 0;
    const uint32_t bytes = uint32_t(nblk) * ((fr ? br : 0u) + (fc ? 2 * br : 0u)) + uint32_t(nrhs) * seg;
    fence_proxy_async_smem();
    if (gfence) fence_proxy_async_global();
    if (bytes == 0) {
      mbar_arrive_u32(bar);
      return;
    }
    mbar_arrive_expect_tx_u32(bar, bytes);
#pragma unroll
    for (int g = 0; g < ng; ++g) {
      int i, kk;
      if (!slot(s, g, i, kk)) continue;
      if (fr) bulk_g2s_u32(dst + uint32_t(g) * slot_r, fr + boff(i, kk, br), br, bar);
      if (fc) bulk_g2s_u32(dst + uint32_t(ng) * slot_r + uint32_t(g) * slot_c, fc + boff(i, kk, 2 * br), 2 * br, bar);
    }
    if (rrow) {
      uint32_t r = dst + rhs_at;
      const size_t o = size_t(s) * (seg >> 3);
      if (x0) { bulk_g2s_u32(r, x0 + o, seg, bar); r += seg; }
      if (x1) { bulk_g2s_u32(r, x1 + o, seg, bar); r += seg; }
      if (xre) {
        bulk_g2s_u32(r, xre + o, seg, bar);
        bulk_g2s_u32(r + seg, xim + o, seg, bar);
      }
    }
  }
};

// a += sum_m col[m nv] x[m] with independent accumulators (col: shared,
// transposed block).  With FP32 factors the sweep accumulates in FP32: the
// factor's own rounding is of the same order, and the FP64 Newton residual
// corrects whatever the preconditioner apply leaves.
// With nv a multiple of 4 (x then 16-byte aligned in the ring) x is read in
// 16-byte vectors, one broadcast load per four products; the sums are the
// same either way.
__device__ __forceinline__ void col_dot(const float* col, const float* x, int nv, float& a) {
  float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
  int m = 0;
  if ((nv & 3) == 0) {
    for (; m < nv; m += 4) {
      const float4 xv = *reinterpret_cast<const float4*>(x + m);
      a0 = fmaf(col[m * nv], xv.x, a0);
      a1 = fmaf(col[(m + 1) * nv], xv.y, a1);
      a2 = fmaf(col[(m + 2) * nv], xv.z, a2);
      a3 = fmaf(col[(m + 3) * nv], xv.w, a3);
    }
  } else {
    for (; m + 3 < nv; m += 4) {
      a0 = fmaf(col[m * nv], x[m], a0);
      a1 = fmaf(col[(m + 1) * nv], x[m + 1], a1);
      a2 = fmaf(col[(m + 2) * nv], x[m + 2], a2);
      a3 = fmaf(col[(m + 3) * nv], x[m + 3], a3);
    }
    for (; m < nv; ++m) a0 = fmaf(col[m * nv], x[m], a0);
  }
  a += (a0 + a1) + (a2 + a3);
}
__device__ __forceinline__ void col_dot_c(const Cx<float>* col, const float* xr, const float* xi, int nv, float& ar,
                                          float& ai) {
  float r0 = 0.f, r1 = 0.f, i0 = 0.f, i1 = 0.f;
  int m = 0;
  if ((nv & 3) == 0) {
    for (; m < nv; m += 4) {
      const float4 xr4 = *reinterpret_cast<const float4*>(xr + m);
      const float4 xi4 = *reinterpret_cast<const float4*>(xi + m);
      const Cx<float> b0 = col[m * nv], b1 = col[(m + 1) * nv], b2 = col[(m + 2) * nv], b3 = col[(m + 3) * nv];
      r0 = fmaf(b0.re, xr4.x, r0);
      r0 = fmaf(-b0.im, xi4.x, r0);
      i0 = fmaf(b0.re, xi4.x, i0);
      i0 = fmaf(b0.im, xr4.x, i0);
      r1 = fmaf(b1.re, xr4.y, r1);
      r1 = fmaf(-b1.im, xi4.y, r1);
      i1 = fmaf(b1.re, xi4.y, i1);
      i1 = fmaf(b1.im, xr4.y, i1);
      r0 = fmaf(b2.re, xr4.z, r0);
      r0 = fmaf(-b2.im, xi4.z, r0);
      i0 = fmaf(b2.re, xi4.z, i0);
      i0 = fmaf(b2.im, xr4.z, i0);
      r1 = fmaf(b3.re, xr4.w, r1);
      r1 = fmaf(-b3.im, xi4.w, r1);
      i1 = fmaf(b3.re, xi4.w, i1);
      i1 = fmaf(b3.im, xr4.w, i1);
    }
  }
  for (; m + 1 < nv; m += 2) {
    const Cx<float> b0 = col[m * nv], b1 = col[(m + 1) * nv];
    r0 = fmaf(b0.re, xr[m], r0);
    r0 = fmaf(-b0.im, xi[m], r0);
    i0 = fmaf(b0.re, xi[m], i0);
    i0 = fmaf(b0.im, xr[m], i0);
    r1 = fmaf(b1.re, xr[m + 1], r1);
    r1 = fmaf(-b1.im, xi[m + 1], r1);
    i1 = fmaf(b1.re, xi[m + 1], i1);
    i1 = fmaf(b1.im, xr[m + 1], i1);
  }
  if (m < nv) {
    const Cx<float> b0 = col[m * nv];
    r0 = fmaf(b0.re, xr[m], r0);
    r0 = fmaf(-b0.im, xi[m], r0);
    i0 = fmaf(b0.re, xi[m], i0);
    i0 = fmaf(b0.im, xr[m], i0);
  }
  ar += r0 + r1;
  ai += i0 + i1;
}
__device__ __forceinline__ void col_dot(const float* col, const double* x, int nv, double& a) {
  double a0 = 0.0, a1 = 0.0;
  int m = 0;
  for (; m + 1 < nv; m += 2) {
    a0 = fma(double(col[m * nv]), x[m], a0);
    a1 = fma(double(col[(m + 1) * nv]), x[m + 1], a1);
  }
  if (m < nv) a0 = fma(double(col[m * nv]), x[m], a0);
  a += a0 + a1;
}
__device__ __forceinline__ void col_dot(const double* col, const double* x, int nv, double& a) {
  double a0 = 0.0, a1 = 0.0;
  int m = 0;
  for (; m + 1 < nv; m += 2) {
    a0 = fma(col[m * nv], x[m], a0);
    a1 = fma(col[(m + 1) * nv], x[m + 1], a1);
  }
  if (m < nv) a0 = fma(col[m * nv], x[m], a0);
  a += a0 + a1;
}
template <typename T>
__device__ __forceinline__ void col_dot_c(const Cx<T>* col, const double* xr, const double* xi, int nv, double& ar,
                                          double& ai) {  // FP64 accumulation
  double r0 = 0.0, i0 = 0.0;
  for (int m = 0; m < nv; ++m) {
    const Cx<T> b = col[m * nv];
    const double br = double(b.re), bi = double(b.im);
    r0 = fma(br, xr[m], r0);
    r0 = fma(-bi, xi[m], r0);
    i0 = fma(br, xi[m], i0);
    i0 = fma(bi, xr[m], i0);
  }
  ar += r0;
  ai += i0;
}

// What slot g of block row i multiplies: forward rows take L_{i,i-bw+g}
// (g < bw) times the solved segment i - bw + g into the L sum, and P^-1_{i-1}
// (g = bw) times segment i - 1 into z; backward rows take W_{i,i+1+g} (g < bw)
// times segment i + 1 + g.  valid: the row has that block.
struct StageSlot {
  int seg;
  bool valid, to_z;
};
template <int BW>
__device__ __forceinline__ StageSlot stage_slot(bool fwd, int i, int ns, int g) {
  StageSlot q;
  if (fwd) {
    q.to_z = g >= BW;
    q.seg = q.to_z ? i - 1 : i - BW + g;
    q.valid = q.to_z ? i >= 1 : (i < ns && q.seg >= 0);
  } else {
    q.to_z = false;
    q.seg = i + 1 + g;
    q.valid = g < BW && q.seg < ns;
  }
  return q;
}

// Returns false when a bounded wait gave up (the solve result is then invalid
// and *P.err is set).  `phase` holds the parity bits of the nbuf barriers and
// is carried across calls (a sweep leaves every barrier with an even number
// of completed phases or not: each thread tracks them); every thread of the
// CTA calls this.
// BW: the factor's off-diagonal blocks per side (3 or 7), a template
// parameter so that the per-stage block loops unroll.
template <typename FT, int BW>
__device__ __noinline__ bool blu_solve_staged_bw(const SolveSet<FT>& S, const SolveStage& P,
                                                    uint32_t& phase) {
  if (*P.err) return false;
  // The set's and the stage's members as scalars, read once: the loop below
  // indexes nothing of S or P at run time (see StageCopies).
  const int ns = S.R.nb;  // block rows
  const int nv = S.R.b;   // block size
  const int nr = S.nr, nc = S.nc;
  constexpr int bw = BW;
  constexpr int ng = bw + 1;                // slots per stage
  constexpr int rmask = (bw < 4 ? 4 : 8) - 1;
  const int nstage = 2 * ns + 1;
  const int tid = threadIdx.x;
  // roles: Gr lanes own one row of a real system and Gc lanes one row of the
  // complex system, each lane the slots g = its lane, + G, ... of the stage;
  // real rows first, the complex ones from the next warp boundary, and at
  // least one thread left over to issue the copies where the block allows
  const int nreal = nr * nv;
  const int nthr = int(blockDim.x);
  int Gc = 4;
  while (Gc > 1 && ((nreal + 31) & ~31) + Gc * nv > nthr) Gc >>= 1;
  const int ncthr = nc > 0 ? Gc * nv : 0;
  int Gr = 4;
  while (Gr > 1 && ((nreal * Gr + 31) & ~31) + ncthr > nthr - 1) Gr >>= 1;
  const int cbase = (nreal * Gr + 31) & ~31;
  const bool is_r = tid < nreal * Gr;
  const int rrow = is_r ? tid / Gr : 0, rg = is_r ? tid - rrow * Gr : 0;
  const int rsys = is_r ? rrow / nv : 0;
  const int rj = is_r ? rrow - rsys * nv : 0;
  const bool is_c = nc > 0 && tid >= cbase && tid < cbase + ncthr;
  const int cu = is_c ? tid - cbase : 0;
  const int cj = cu / Gc, cg = cu - cj * Gc;
  double* const xr_me = rsys ? S.xr[1] : S.xr[0];  // this thread's real system's vectors
  double* const zr_me = rsys ? S.zr[1] : S.zr[0];
  double* const xc_re = S.xc_re;
  double* const xc_im = S.xc_im;
  double* const zc_re = S.zc_re;
  double* const zc_im = S.zc_im;
  using RT = FT;  // accumulation / ring type: float with FP32 factors, double with FP64
  // ring segments of rs entries: FP32 segments are padded by four entries, so
  // that the segments which the lanes of a warp read together start in
  // different banks (the ring area is sized for FP64 entries, which this fits)
  const int rs = nv + (sizeof(RT) == 4 ? 4 : 0);
  const int rlen = (rmask + 1) * rs;  // ring length per right-hand-side array
  // stage buffers, ring and z as shared-space pointers (see fpe_dsmem)
  unsigned char* const sbuf0 = fpe_dsmem + dsmem_offset(P.buf[0]);
  const uint32_t sstride = uint32_t(P.buf[1] - P.buf[0]);
  const int slot_r = P.slot_r, slot_c = P.slot_c;
  const bool rhs_bulk = P.rhs_bulk;
  RT* ringb = reinterpret_cast<RT*>(fpe_dsmem + dsmem_offset(P.ring));
  RT* ring_c_re = ringb + nr * rlen;
  RT* ring_c_im = ring_c_re + rlen;
  // z of every block row in shared memory when it fits (real systems first,
  // then the complex re and im parts), else in the global scratch vectors
  const int N = ns * nv;
  const bool zsh = P.zbuf && size_t(nr + 2 * nc) * N * sizeof(RT) <= size_t(P.zcap);
  RT* zs = zsh ? reinterpret_cast<RT*>(fpe_dsmem + dsmem_offset(P.zbuf)) : nullptr;
  RT* zs_re = zs + nr * N;
  RT* zs_im = zs_re + N;
  const int rhs_at = ng * (slot_r + (nc > 0 ? slot_c : 0));  // rhs segments in a stage buffer
  int* const err = P.err;

  // the thread that issues the copies: an idle one when the roles leave one
  const int issuer = (nthr - 1 >= max(nreal * Gr, cbase + ncthr)) ? nthr - 1 : 0;
  const int nbuf = P.nbuf;
  StageCopies<FT, BW> cp;
  if (tid == issuer) {
    cp.fr = nr > 0 ? reinterpret_cast<const unsigned char*>(S.R.F) : nullptr;
    cp.fc = nc > 0 ? reinterpret_cast<const unsigned char*>(S.Cf.F) : nullptr;
    cp.br = uint32_t(S.R.bs) * uint32_t(sizeof(FT));
    cp.nb = ns;
    cp.dst0 = smem_u32(sbuf0);
    cp.dstep = sstride;
    cp.slot_r = uint32_t(slot_r);
    cp.slot_c = uint32_t(slot_c);
    cp.rhs_at = uint32_t(rhs_at);
    cp.bar0 = smem_u32(P.bar);
    cp.seg = uint32_t(nv) * 8u;
    cp.x0 = nr > 0 ? S.xr[0] : nullptr;
    cp.x1 = nr > 1 ? S.xr[1] : nullptr;
    cp.xre = nc > 0 ? xc_re : nullptr;
    cp.xim = nc > 0 ? xc_im : nullptr;
    cp.rhs = rhs_bulk;
  }
  uint32_t pend = 0;  // buffers with a stage in flight (the issuer's view)
  if (tid == issuer) {
    for (int q = 0; q < nbuf && q < nstage; ++q) {
      cp.issue(q, q, q == 0);
      pend |= 1u << q;
    }
  }
  bool ok = true;
  // the barriers' parity bits and the timers stay in registers during the sweep
  uint32_t ph = phase;
  long long t_wait = 0, t_work = 0, t_bar = 0;
  unsigned long long* const bars = P.bar;
  const long long wlim = P.wait_limit;
  int b = 0;  // buffer of stage s: s mod nbuf
  for (int s = 0; s < nstage; ++s, b = (b + 1 == nbuf) ? 0 : b + 1) {
    const long long tw0 = clock64();
    const bool landed = mbar_wait_bounded(bars + b, (ph >> b) & 1u, wlim);
    t_wait += clock64() - tw0;
    if (landed) {
      ph ^= 1u << b;
      pend &= ~(1u << b);
    } else {
      ok = false;
      *err = 1;
    }
    ok = __all_sync(0xffffffffu, ok);  // uniform per warp before the group shuffles
    const unsigned char* buf = sbuf0 + b * sstride;
    const bool fwd = s <= ns;
    const int i = fwd ? s : 2 * ns - s;
    if (ok) {
      RT a = RT(0), z = RT(0);  // real row: L products (forward) or W products, and P^-1 y
      // the row's right-hand side (forward) or z (backward), loaded before the products
      double xb = 0.0;
      if (is_r && rg == 0) {
        if (fwd) {
          if (i < ns) xb = rhs_bulk ? reinterpret_cast<const double*>(buf + rhs_at)[rsys * nv + rj] : xr_me[i * nv + rj];
        } else {
          xb = zsh ? double(zs[rsys * N + i * nv + rj]) : zr_me[i * nv + rj];
        }
      }
      if (is_r) {
        // one code path for every slot (the lanes of a warp hold different
        // slots and stay converged): the slot's ring segment, and whether it
        // feeds the L / W sum or P^-1 y
        const RT* ring = ringb + rsys * rlen;
        for (int g = rg; g < ng; g += Gr) {
          const StageSlot q = stage_slot<bw>(fwd, i, ns, g);
          if (q.valid) {
            RT d = RT(0);
            col_dot(reinterpret_cast<const FT*>(buf + g * slot_r) + rj, ring + (q.seg & rmask) * rs, nv, d);
            if (q.to_z) z += d;
            else a += d;
          }
        }
      }
      if (tid < cbase) {  // group reduction over the Gr lanes of a real row (real warps only)
        for (int o = Gr >> 1; o > 0; o >>= 1) {
          a += __shfl_down_sync(0xffffffffu, a, o, Gr);
          z += __shfl_down_sync(0xffffffffu, z, o, Gr);
        }
      }
      if (is_r && rg == 0) {
        if (fwd) {
          if (i < ns) ringb[rsys * rlen + (i & rmask) * rs + rj] = RT(xb - double(a));
          if (i >= 1) {
            if (zsh) zs[rsys * N + (i - 1) * nv + rj] = z;
            else zr_me[(i - 1) * nv + rj] = double(z);
          }
        } else {
          const double x = xb - double(a);
          ringb[rsys * rlen + (i & rmask) * rs + rj] = RT(x);
          xr_me[i * nv + rj] = x;
        }
      }
      RT ar = RT(0), ai = RT(0), zr = RT(0), zi = RT(0);
      // the row's right-hand side (forward) or z (backward), loaded before the products
      double cre = 0.0, cim = 0.0;
      if (is_c && cg == 0) {
        if (!fwd) {
          cre = zsh ? double(zs_re[i * nv + cj]) : zc_re[i * nv + cj];
          cim = zsh ? double(zs_im[i * nv + cj]) : zc_im[i * nv + cj];
        } else if (i < ns) {
          if (rhs_bulk) {
            const double* rb = reinterpret_cast<const double*>(buf + rhs_at) + nr * nv;
            cre = rb[cj];
            cim = rb[nv + cj];
          } else {
            cre = xc_re[i * nv + cj];
            cim = xc_im[i * nv + cj];
          }
        }
      }
      if (is_c) {
        const unsigned char* cb = buf + ng * slot_r;
        for (int g = cg; g < ng; g += Gc) {
          const StageSlot q = stage_slot<bw>(fwd, i, ns, g);
          if (q.valid) {
            RT dr = RT(0), di = RT(0);
            const int seg = (q.seg & rmask) * rs;
            col_dot_c(reinterpret_cast<const Cx<FT>*>(cb + g * slot_c) + cj, ring_c_re + seg, ring_c_im + seg, nv, dr,
                      di);
            if (q.to_z) {
              zr += dr;
              zi += di;
            } else {
              ar += dr;
              ai += di;
            }
          }
        }
      }
      // group reduction over the Gc lanes of a complex row (complex warps only)
      if (tid >= cbase) {
        for (int o = Gc >> 1; o > 0; o >>= 1) {
          ar += __shfl_down_sync(0xffffffffu, ar, o, Gc);
          ai += __shfl_down_sync(0xffffffffu, ai, o, Gc);
          zr += __shfl_down_sync(0xffffffffu, zr, o, Gc);
          zi += __shfl_down_sync(0xffffffffu, zi, o, Gc);
        }
      }
      if (is_c && cg == 0) {
        if (fwd) {
          if (i < ns) {
            ring_c_re[(i & rmask) * rs + cj] = RT(cre - double(ar));
            ring_c_im[(i & rmask) * rs + cj] = RT(cim - double(ai));
          }
          if (i >= 1) {
            if (zsh) {
              zs_re[(i - 1) * nv + cj] = zr;
              zs_im[(i - 1) * nv + cj] = zi;
            } else {
              zc_re[(i - 1) * nv + cj] = double(zr);
              zc_im[(i - 1) * nv + cj] = double(zi);
            }
          }
        } else {
          const double xr = cre - double(ar), xi = cim - double(ai);
          ring_c_re[(i & rmask) * rs + cj] = RT(xr);
          ring_c_im[(i & rmask) * rs + cj] = RT(xi);
          xc_re[i * nv + cj] = xr;
          xc_im[i * nv + cj] = xi;
        }
      }
    }
    const long long tb0 = clock64();
    t_work += tb0 - tw0;
    // the stage barrier also tells every thread whether a wait gave up (the
    // failing threads set *P.err, which the caller reads after the sweep)
    const bool failed = __syncthreads_or(ok ? 0 : 1) != 0;
    t_bar += clock64() - tb0;
    if (failed) {
      ok = false;
      break;
    }
    if (tid == issuer && s + nbuf < nstage) {
      cp.issue(s + nbuf, b, false);
      pend |= 1u << b;
    }
  }
  if (!ok && tid == issuer) {
    // let copies still in flight land before the buffers are reused: the full
    // (about one second) limit, whatever the stage waits were given
    for (int q = 0; q < nbuf; ++q)
      if ((pend >> q) & 1u) mbar_wait_bounded(bars + q, (ph >> q) & 1u, kBulkWaitLimit);
  }
  phase = ph;
  *P.wait_cycles += t_wait;
  *P.work_cycles += t_work;
  *P.bar_cycles += t_bar;
  __syncthreads();
  return ok;
}

template <typename FT>
__device__ __forceinline__ bool blu_solve_staged(const SolveSet<FT>& S, const SolveStage& P, uint32_t& phase) {
  const int bw = S.R.bw;
  return bw == 7 ? blu_solve_staged_bw<FT, 7>(S, P, phase) : blu_solve_staged_bw<FT, 3>(S, P, phase);
}

}  // namespace fpe
