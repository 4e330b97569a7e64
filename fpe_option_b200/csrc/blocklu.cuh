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

// Gauss-Jordan inverse with partial pivoting of the nv x nv block P (global,
// in place).  aug: nv x 2nv shared ET; aux: 6 nv shared ET.
template <typename ET>
__device__ bool gj_invert(ET* P, int nv, ET* aug, ET* aux, int* piv_s) {
  using A = typename AccOf<ET>::T;
  const int w = 2 * nv;
  for (int e = threadIdx.x; e < nv * w; e += blockDim.x) {
    const int r = e / w, c = e - r * w;
    if (c < nv) aug[e] = P[r * nv + c];
    else st_elem(aug[e], (c - nv == r) ? aone(A()) : azero(A()));
  }
  __syncthreads();
  ET* prow = aux;
  ET* orow = aux + w;
  ET* fcol = aux + 2 * w;
  bool ok = true;
  for (int c = 0; c < nv; ++c) {
    if (threadIdx.x < 32) {
      double best = -1.0;
      int bi = c;
      for (int r = c + threadIdx.x; r < nv; r += 32) {
        const double v = amag(acc_load(aug[r * w + c]));
        if (v > best) {
          best = v;
          bi = r;
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
      if (threadIdx.x == 0) piv_s[0] = bi;
    }
    __syncthreads();
    const int p = piv_s[0];
    const A pv = acc_load(aug[p * w + c]);
    if (amag(pv) == 0.0) ok = false;
    const A inv = ainv(pv);
    for (int l = threadIdx.x; l < w; l += blockDim.x) {
      st_elem(prow[l], amul(acc_load(aug[p * w + l]), inv));
      orow[l] = aug[c * w + l];
    }
    for (int r = threadIdx.x; r < nv; r += blockDim.x) fcol[r] = (r == p) ? aug[c * w + c] : aug[r * w + c];
    __syncthreads();
    for (int e = threadIdx.x; e < nv * w; e += blockDim.x) {
      const int r = e / w, l = e - r * w;
      if (r == c) {
        aug[e] = prow[l];
      } else {
        const A src = acc_load((r == p) ? orow[l] : aug[e]);
        st_elem(aug[e], asub(src, amul(acc_load(fcol[r]), acc_load(prow[l]))));
      }
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < nv * nv; e += blockDim.x) {
    const int r = e / nv, c = e - r * nv;
    P[e] = aug[r * w + nv + c];
  }
  __syncthreads();
  return ok;
}

// Factor in place.  sbig: shared scratch of max(3 nv^2, 2 nv^2 + 6 nv) ET.
template <typename ET>
__device__ bool blu_factor(const BlockLU<ET>& L, ET* sbig, int* piv_s) {
  using A = typename AccOf<ET>::T;
  const int ns = L.ns, nv = L.nv, nn = nv * nv;
  bool ok = true;
  for (int i = 0; i < ns; ++i) {
    ET* P = L.blk(i, 3);
    ok &= gj_invert<ET>(P, nv, sbig, sbig + 2 * nn, piv_s);
    const int nr = min(i + 3, ns - 1) - i;
    if (nr > 0) {
      // L_ri = E_ri P_i^-1 -> shared
      for (int e = threadIdx.x; e < nr * nn; e += blockDim.x) {
        const int rr = e / nn, jl = e - rr * nn, j = jl / nv, l = jl - j * nv;
        const ET* E = L.blk(i + 1 + rr, 2 - rr);
        A acc = azero(A());
        for (int m = 0; m < nv; ++m) afma(acc, acc_load(E[j * nv + m]), acc_load(P[m * nv + l]));
        st_elem(sbig[e], acc);
      }
      __syncthreads();
      for (int e = threadIdx.x; e < nr * nn; e += blockDim.x) {
        const int rr = e / nn, jl = e - rr * nn;
        L.blk(i + 1 + rr, 2 - rr)[jl] = sbig[e];
      }
      // E_rc -= L_ri U_ic for r, c in (i, i + 3]
      for (int e = threadIdx.x; e < nr * nr * nn; e += blockDim.x) {
        const int rc2 = e / nn, jl = e - rc2 * nn;
        const int rr = rc2 / nr, cc = rc2 - rr * nr;
        const int r = i + 1 + rr, c = i + 1 + cc;
        const int j = jl / nv, l = jl - j * nv;
        const ET* Lr = sbig + rr * nn + j * nv;
        const ET* U = L.blk(i, c - i + 3);
        A acc = azero(A());
        for (int m = 0; m < nv; ++m) afma(acc, acc_load(Lr[m]), acc_load(U[m * nv + l]));
        ET* E = L.blk(r, c - r + 3);
        st_elem(E[jl], asub(acc_load(E[jl]), acc));
      }
      __syncthreads();
      // W_ik = P_i^-1 U_ik (in place via shared staging)
      for (int e = threadIdx.x; e < nr * nn; e += blockDim.x) {
        const int cc = e / nn, jl = e - cc * nn, j = jl / nv, l = jl - j * nv;
        const ET* U = L.blk(i, 4 + cc);
        A acc = azero(A());
        for (int m = 0; m < nv; ++m) afma(acc, acc_load(P[j * nv + m]), acc_load(U[m * nv + l]));
        st_elem(sbig[e], acc);
      }
      __syncthreads();
      for (int e = threadIdx.x; e < nr * nn; e += blockDim.x) {
        const int cc = e / nn, jl = e - cc * nn;
        L.blk(i, 4 + cc)[jl] = sbig[e];
      }
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
