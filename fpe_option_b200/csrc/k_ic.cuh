// Nonnegative initial-condition projection, one CTA per solve.
//
// Reference: initial_condition_from_cached (src/engines/fpe/initial_cond.mojo:70-131):
//   b  = (Bs (x) Bv)^T W delta            (truncated bivariate normal, :25-67)
//   A  = D^-1 M D^-1,  solve min 1/2|A c - D^-1 b|^2 + lam/2 |c|^2, c >= 0 by
//        ADMM (src/numerics/optim/osqp.mojo:52-159: rho 0.1, sigma 1e-6,
//        lam 1e-6, eps 1e-8, <= 50000 iterations, KKT = A^T A + (lam+sigma+rho) I)
//   q0 = max(D^-1 c, 0) / (m^T q0),  m = (Bs (x) Bv)^T W 1
// Here A = As (x) Av is Kronecker, so the KKT matrix As^2 (x) Av^2 + alpha I
// is diagonalised by the eigenvectors of As and Av (cyclic Jacobi on the
// device); each ADMM x-update is four small dense products instead of a
// sparse LU solve.  On the reference discretization the iteration is the
// reference's; the config discretization adds residual balancing of rho and
// over-relaxation (both below).
#pragma once
#include "dev_common.cuh"

namespace fpe {

// C[m x n] = op(A) op(B) with element (r, p) of op(A) at A[r*ar + p*ac] and
// element (p, c) of op(B) at B[p*br + c*bc].
__device__ void cta_gemm(int m, int n, int k, const double* __restrict__ A, int ar, int ac,
                         const double* __restrict__ B, int br, int bc, double* __restrict__ C,
                         int ldc) {
  for (int e = threadIdx.x; e < m * n; e += blockDim.x) {
    const int r = e / n, c = e - r * n;
    double acc = 0.0;
    for (int p = 0; p < k; ++p) acc += A[r * ar + p * ac] * B[p * br + c * bc];
    C[r * ldc + c] = acc;
  }
}

// Same product with two adjacent outputs per thread (shared-memory operands);
// when scale is given the result is multiplied elementwise by it.
__device__ void cta_gemm2(int m, int n, int k, const double* __restrict__ A, int ar, int ac,
                          const double* __restrict__ B, int br, int bc, double* __restrict__ C,
                          int ldc, const double* __restrict__ scale) {
  const int n2 = (n + 1) / 2;
  for (int e = threadIdx.x; e < m * n2; e += blockDim.x) {
    const int r = e / n2, c = 2 * (e - r * n2);
    const int c1 = c + 1 < n ? c + 1 : c;
    double a0 = 0.0, a1 = 0.0;
    for (int p = 0; p < k; ++p) {
      const double av = A[r * ar + p * ac];
      a0 = fma(av, B[p * br + c * bc], a0);
      a1 = fma(av, B[p * br + c1 * bc], a1);
    }
    if (scale) {
      a0 *= scale[r * ldc + c];
      a1 *= scale[r * ldc + c1];
    }
    C[r * ldc + c] = a0;
    if (c + 1 < n) C[r * ldc + c + 1] = a1;
  }
}

// C[m x n] = op(A) B (.* scale) with a 2 x 4 register tile per thread:
// element (r, p) of op(A) at A[r*ar + p*ac]; B row-major with row stride ldb.
// When vec is set (ldb even, B 16-byte aligned) a tile row of B is two
// 16-byte loads.  Consecutive threads take consecutive column tiles, so a
// warp reads contiguous rows of B.
__device__ void cta_gemm24(int m, int n, int k, const double* __restrict__ A, int ar, int ac,
                           const double* __restrict__ B, int ldb, double* __restrict__ C, int ldc,
                           const double* __restrict__ scale, bool vec) {
  const int mt = (m + 1) / 2, nt = (n + 3) / 4;
  for (int t = threadIdx.x; t < mt * nt; t += blockDim.x) {
    const int ti = t / nt, tj = t - ti * nt;
    const int r0 = 2 * ti, r1 = r0 + 1 < m ? r0 + 1 : r0;
    const int c0 = 4 * tj;
    const double* a0 = A + r0 * ar;
    const double* a1 = A + r1 * ar;
    double acc0[4] = {0.0, 0.0, 0.0, 0.0}, acc1[4] = {0.0, 0.0, 0.0, 0.0};
    if (vec && c0 + 3 < n) {
#pragma unroll 4
      for (int p = 0; p < k; ++p) {
        const double x0 = a0[p * ac], x1 = a1[p * ac];
        const double2 b01 = *reinterpret_cast<const double2*>(B + p * ldb + c0);
        const double2 b23 = *reinterpret_cast<const double2*>(B + p * ldb + c0 + 2);
        acc0[0] = fma(x0, b01.x, acc0[0]);
        acc0[1] = fma(x0, b01.y, acc0[1]);
        acc0[2] = fma(x0, b23.x, acc0[2]);
        acc0[3] = fma(x0, b23.y, acc0[3]);
        acc1[0] = fma(x1, b01.x, acc1[0]);
        acc1[1] = fma(x1, b01.y, acc1[1]);
        acc1[2] = fma(x1, b23.x, acc1[2]);
        acc1[3] = fma(x1, b23.y, acc1[3]);
      }
    } else {
      for (int p = 0; p < k; ++p) {
        const double x0 = a0[p * ac], x1 = a1[p * ac];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const double b = c0 + j < n ? B[p * ldb + c0 + j] : 0.0;
          acc0[j] = fma(x0, b, acc0[j]);
          acc1[j] = fma(x1, b, acc1[j]);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = c0 + j;
      if (c >= n) break;
      double v0 = acc0[j], v1 = acc1[j];
      if (scale) {
        v0 *= scale[r0 * ldc + c];
        v1 *= scale[r1 * ldc + c];
      }
      C[r0 * ldc + c] = v0;
      if (r1 != r0) C[r1 * ldc + c] = v1;
    }
  }
}

// Cyclic Jacobi eigendecomposition of the symmetric n x n matrix A (row-major,
// destroyed; eigenvalues left on its diagonal), eigenvectors in the columns
// of V.  Round-robin ordering: n/2 disjoint rotations per round.
__device__ void jacobi_eig(int n, double* A, double* V, double* cs_s, double* red) {
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) V[e] = (e / n == e % n) ? 1.0 : 0.0;
  __syncthreads();
  const int m = n + (n & 1);
  const int half = m / 2;
  double norm2 = 0.0;
  {
    double s = 0.0;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) s += A[e] * A[e];
    norm2 = block_sum1(s, red);
  }
  for (int sweep = 0; sweep < 40; ++sweep) {
    double off = 0.0;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x)
      if (e / n != e % n) off += A[e] * A[e];
    off = block_sum1(off, red);
    if (off <= 1e-30 * norm2 || off == 0.0) break;
    for (int r = 0; r < m - 1; ++r) {
      // pair k: (a, b) with the circle method
      for (int k = threadIdx.x; k < half; k += blockDim.x) {
        int a, b;
        if (k == 0) {
          a = r % (m - 1);
          b = m - 1;
        } else {
          a = (r + k) % (m - 1);
          b = (r - k + (m - 1)) % (m - 1);
        }
        if (a > b) {
          int t = a;
          a = b;
          b = t;
        }
        double c = 1.0, s = 0.0;
        if (b < n) {
          double apq = A[a * n + b];
          if (fabs(apq) > 1e-300) {
            double tau = (A[b * n + b] - A[a * n + a]) / (2.0 * apq);
            double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
          }
        }
        cs_s[4 * k + 0] = c;
        cs_s[4 * k + 1] = s;
        cs_s[4 * k + 2] = a;
        cs_s[4 * k + 3] = b;
      }
      __syncthreads();
      // columns: A <- A J, V <- V J
      for (int e = threadIdx.x; e < half * n; e += blockDim.x) {
        const int k = e / n, row = e - k * n;
        const int a = int(cs_s[4 * k + 2]), b = int(cs_s[4 * k + 3]);
        if (b >= n) continue;
        const double c = cs_s[4 * k], s = cs_s[4 * k + 1];
        double x = A[row * n + a], y = A[row * n + b];
        A[row * n + a] = c * x - s * y;
        A[row * n + b] = s * x + c * y;
        x = V[row * n + a];
        y = V[row * n + b];
        V[row * n + a] = c * x - s * y;
        V[row * n + b] = s * x + c * y;
      }
      __syncthreads();
      // rows: A <- J^T A
      for (int e = threadIdx.x; e < half * n; e += blockDim.x) {
        const int k = e / n, col = e - k * n;
        const int a = int(cs_s[4 * k + 2]), b = int(cs_s[4 * k + 3]);
        if (b >= n) continue;
        const double c = cs_s[4 * k], s = cs_s[4 * k + 1];
        double x = A[a * n + col], y = A[b * n + col];
        A[a * n + col] = c * x - s * y;
        A[b * n + col] = s * x + c * y;
      }
      __syncthreads();
    }
  }
}

// Value of recombined dof c at x (sum of its original B-splines, 1e-12 drop).
__device__ double recombined_value(const double* t, int nt, double x, int c, bool lneu, bool rneu) {
  const int nb = nt - 4, rc = nb - 2;
  double v = 0.0;
  auto add = [&](int o) {
    double b = bs_value(t, nt, x, o, 3);
    if (b > 1e-12 || b < -1e-12) v += b;
  };
  if (c == 0 && lneu && rc > 0) add(0);
  add(c + 1);
  if (c == rc - 1 && rneu && rc > 0) add(nb - 1);
  return v;
}

// Integral of a normal density against recombined dof c over its support,
// ic_sub equal subintervals per knot span, textbook 4-point Gauss-Legendre.
__device__ double gauss_moment(const double* t, int nt, int c, bool lneu, bool rneu, double off,
                               double jac, double mean, double sd, int ic_sub) {
  const int nb = nt - 4, rc = nb - 2;
  int omin = c + 1, omax = c + 1;
  if (c == 0 && lneu && rc > 0) omin = 0;
  if (c == rc - 1 && rneu && rc > 0) omax = nb - 1;
  double glx[4], glw[4];
  {
    double a = sqrt(3.0 / 7.0 - 2.0 / 7.0 * sqrt(6.0 / 5.0));
    double b = sqrt(3.0 / 7.0 + 2.0 / 7.0 * sqrt(6.0 / 5.0));
    double wa = (18.0 + sqrt(30.0)) / 36.0, wb = (18.0 - sqrt(30.0)) / 36.0;
    glx[0] = -b; glx[1] = -a; glx[2] = a; glx[3] = b;
    glw[0] = wb; glw[1] = wa; glw[2] = wa; glw[3] = wb;
  }
  const double nrm = 1.0 / (sqrt(2.0 * CUDART_PI) * sd);
  double acc = 0.0;
  for (int m = omin; m <= omax + 3 && m + 1 < nt; ++m) {
    double a = t[m], b = t[m + 1];
    if (!(b > a)) continue;
    for (int s = 0; s < ic_sub; ++s) {
      double sa = a + (b - a) * double(s) / ic_sub, sb = a + (b - a) * double(s + 1) / ic_sub;
      double mid = 0.5 * (sa + sb), hw = 0.5 * (sb - sa);
      for (int g = 0; g < 4; ++g) {
        double x = mid + hw * glx[g];
        double bv = recombined_value(t, nt, x, c, lneu, rneu);
        if (bv == 0.0) continue;
        double z = (off + x * jac - mean) / sd;
        acc += bv * (nrm * exp(-0.5 * z * z) * (hw * glw[g] * jac));
      }
    }
  }
  return acc;
}

struct IcSmem {
  double red[32 * 8];
  double cs[4 * 96];
};

__global__ void __launch_bounds__(FPE_BLOCK, 1) k_ic(const FpeSolveDesc* __restrict__ descs,
                                                  double* __restrict__ darena,
                                                  int32_t* __restrict__ iarena, int32_t* __restrict__ infos,
                                                  size_t dyn_bytes) {
  __shared__ IcSmem S;
  extern __shared__ __align__(16) unsigned char ic_dyn[];
  const FpeSolveDesc d = descs[blockIdx.x];
  const FpeDLayout DL = fpe_dlayout(d);
  const FpeILayout IL = fpe_ilayout(d);
  double* D = darena + d.off_d;
  int32_t* I = iarena + d.off_i;
  int32_t* info = infos + size_t(blockIdx.x) * FPE_INFO_COUNT;
  if (info[FPE_INFO_STATUS] != 0) return;
  const int nds = info[FPE_INFO_NDOF_S], ndv = info[FPE_INFO_NDOF_V];
  const int N = nds * ndv;
  const double* Ds = D + DL.D_s;
  const double* Dv = D + DL.D_v;
  double* proj = D + DL.proj;

  // ---- projection b -------------------------------------------------------
  if (d.disc == 0) {
    // initial_cond.mojo:25-67: s_sigma = 0.1, v_sigma = 0.1 / (Smax - Smin), rho 0
    const double sigma0 = 0.1;
    const double span = d.smax - d.smin;
    double ss = sigma0, vs = span > 0.0 ? sigma0 / span : sigma0;
    if (ss <= 0.0) ss = 1e-3;
    if (vs <= 0.0) vs = 1e-3;
    const double norm = 1.0 / (2.0 * CUDART_PI * ss * vs * sqrt(1.0));
    const double inv2 = 0.5 / 1.0;
    const double* qws = D + DL.qw_s;
    const double* qps = D + DL.qp_s;
    const double* qwv = D + DL.qw_v;
    const double* qpv = D + DL.qp_v;
    const double* Bs = D + DL.B_s;
    const double* Bv = D + DL.B_v;
    const int32_t* c0s = I + IL.c0_s;
    const int32_t* c0v = I + IL.c0_v;
    const int32_t* rs = I + IL.rng_s;
    const int32_t* rv = I + IL.rng_v;
    for (int e = threadIdx.x; e < N; e += blockDim.x) {
      const int a = e / ndv, b = e - a * ndv;
      double acc = 0.0;
      for (int p = rs[2 * a]; p < rs[2 * a + 1]; ++p) {
        const int la = a - c0s[p];
        if (la < 0 || la > 3) continue;
        const double ba = Bs[4 * p + la];
        if (ba == 0.0) continue;
        const double dsn = (qps[p] - d.S0) / ss, ds2 = dsn * dsn;
        if (ds2 > 50.0) continue;
        double inner = 0.0;
        for (int q = rv[2 * b]; q < rv[2 * b + 1]; ++q) {
          const int lb = b - c0v[q];
          if (lb < 0 || lb > 3) continue;
          const double dvn = (qpv[q] - d.V0) / vs;
          const double z = ds2 + dvn * dvn;
          if (z * inv2 > 50.0) continue;
          double val = norm * exp(-z * inv2);
          if (val < 1e-6) continue;
          inner += Bv[4 * q + lb] * ((qws[p] * qwv[q]) * val);
        }
        acc += ba * inner;
      }
      proj[e] = acc;
    }
  } else {
    // separable wide normal: b = bs (x) bv on a refined quadrature
    const double* ks = D + DL.knot_s;
    const double* kv = D + DL.knot_v;
    const int nks = info[FPE_INFO_NKNOT_S], nkv = info[FPE_INFO_NKNOT_V];
    double* tmp = D + DL.work;  // nds + ndv
    for (int c = threadIdx.x; c < nds + ndv; c += blockDim.x) {
      if (c < nds)
        tmp[c] = gauss_moment(ks, nks, c, d.left_neu != 0, d.right_neu != 0, d.smin,
                              d.smax - d.smin, d.S0, d.ic_sigma_s, d.ic_sub);
      else
        tmp[c] = gauss_moment(kv, nkv, c - nds, true, true, 0.0, 1.0, d.V0, d.ic_sigma_v,
                              d.ic_sub);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < N; e += blockDim.x) {
      const int a = e / ndv, b = e - a * ndv;
      proj[e] = tmp[a] * tmp[nds + b];
    }
  }
  __syncthreads();

  // ---- eigendecomposition of As and Av ----------------------------------
  const double* os = D + DL.op_s;  // As = op_s[0]
  const double* ov = D + DL.op_v;  // Av = op_v[0]
  double* W = D + DL.work;
  double* As = W;
  double* Vs = As + nds * nds;
  double* Av = Vs + nds * nds;
  double* Vv = Av + ndv * ndv;
  double* vec = Vv + ndv * ndv;
  double* x = vec;
  double* z = x + N;
  double* u = z + N;
  double* q = u + N;
  double* rhs = q + N;
  double* t1 = rhs + N;
  double* lam = t1 + N;  // N: 1 / (ls^2 lv^2 + alpha)
  double* bsc = lam + N;
  for (int e = threadIdx.x; e < nds * nds; e += blockDim.x) {
    const int i = e / nds, k = e - i * nds, dd = k - i + 3;
    As[e] = (dd >= 0 && dd < 7) ? os[i * 7 + dd] : 0.0;
  }
  for (int e = threadIdx.x; e < ndv * ndv; e += blockDim.x) {
    const int j = e / ndv, l = e - j * ndv, dd = l - j + 3;
    Av[e] = (dd >= 0 && dd < 7) ? ov[j * 7 + dd] : 0.0;
  }
  __syncthreads();
  // The eigendecompositions run in shared memory when the dynamic area (sized
  // for the ADMM iterates, not yet in use) holds both matrices and both
  // eigenvector sets: each Jacobi round reads and writes whole rows and
  // columns between barriers, which from the global work area costs an L2
  // round trip per phase.  The results go back to the work area once.
  const size_t jac_bytes = (2 * size_t(nds) * nds + 2 * size_t(ndv) * ndv) * sizeof(double);
  if (jac_bytes <= dyn_bytes && fpe_ic_admm_bytes(nds, ndv) <= dyn_bytes) {
    double* jAs = reinterpret_cast<double*>(ic_dyn);
    double* jVs = jAs + nds * nds;
    double* jAv = jVs + nds * nds;
    double* jVv = jAv + ndv * ndv;
    for (int e = threadIdx.x; e < nds * nds; e += blockDim.x) jAs[e] = As[e];
    for (int e = threadIdx.x; e < ndv * ndv; e += blockDim.x) jAv[e] = Av[e];
    __syncthreads();
    jacobi_eig(nds, jAs, jVs, S.cs, S.red);
    jacobi_eig(ndv, jAv, jVv, S.cs, S.red);
    for (int e = threadIdx.x; e < nds * nds; e += blockDim.x) {
      As[e] = jAs[e];
      Vs[e] = jVs[e];
    }
    for (int e = threadIdx.x; e < ndv * ndv; e += blockDim.x) {
      Av[e] = jAv[e];
      Vv[e] = jVv[e];
    }
    __syncthreads();
  } else {
    jacobi_eig(nds, As, Vs, S.cs, S.red);
    jacobi_eig(ndv, Av, Vv, S.cs, S.red);
  }
  const double sigma = 1e-6, lamreg = 1e-6, eps_abs = 1e-8, eps_rel = 1e-8;
  double rho = 0.1;
  const double alpha = lamreg + sigma + rho;
  for (int e = threadIdx.x; e < N; e += blockDim.x) {
    const int a = e / ndv, b = e - a * ndv;
    const double ls = As[a * nds + a], lv = Av[b * ndv + b];
    lam[e] = 1.0 / ((ls * ls) * (lv * lv) + alpha);
    // IC scaling Dinv = 1/sqrt(diag M) (initial_cond.mojo:84-97)
    bsc[e] = proj[e] / (Ds[a] * Dv[b]);
    x[e] = z[e] = u[e] = 0.0;
  }
  __syncthreads();
  // q = A^T (D^-1 b) with A = As (x) Av (symmetric): q = vec(As Bsc Av), applied
  // with the banded factors (the dense copies now hold eigenvalues).
  for (int e = threadIdx.x; e < N; e += blockDim.x) {
    const int a = e / ndv, b = e - a * ndv;
    double acc = 0.0;
    for (int dd = 0; dd < 7; ++dd) {
      const int l = b + dd - 3;
      if (l >= 0 && l < ndv) acc += ov[b * 7 + dd] * bsc[a * ndv + l];
    }
    t1[e] = acc;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < N; e += blockDim.x) {
    const int a = e / ndv, b = e - a * ndv;
    double acc = 0.0;
    for (int dd = 0; dd < 7; ++dd) {
      const int k = a + dd - 3;
      if (k >= 0 && k < nds) acc += os[a * 7 + dd] * t1[k * ndv + b];
    }
    q[e] = acc;
  }
  __syncthreads();

  // ---- ADMM (osqp.mojo:93-157) ------------------------------------------
  // Shared-memory resident when it fits: eigenvectors Vs, Vv and Vv^T, the
  // five iterates, lam and q, each section at an even (16-byte) offset.  In
  // shared memory the rows of Vs and of the intermediate t1 are padded by two
  // doubles (strides lds, ldt): three of the four products read their left
  // operand along rows, and unpadded rows of 32 or 64 doubles put a warp's
  // four row groups on one bank.
  const size_t need = fpe_ic_admm_bytes(nds, ndv);
  int lds = nds, ldt = ndv;
  double* sVs = Vs;
  double* sVv = Vv;
  double* sVvT = vec + 8 * size_t(N);  // global fallback: after the iterates (work area)
  double *sx = x, *sz = z, *su = u, *sq = q, *srhs = rhs, *st1 = t1, *slam = lam;
  auto ev = [](int n) { return (n + 1) & ~1; };
  if (need <= dyn_bytes) {
    double* sm = reinterpret_cast<double*>(ic_dyn);
    lds = nds + 2;
    ldt = ndv + 2;
    sVs = sm;
    sVv = sVs + ev(nds * lds);
    sVvT = sVv + ev(ndv * ndv);
    sx = sVvT + ev(ndv * ndv);
    sz = sx + ev(N);
    su = sz + ev(N);
    sq = su + ev(N);
    srhs = sq + ev(N);
    st1 = srhs + ev(N);
    slam = st1 + ev(nds * ldt);
    for (int e = threadIdx.x; e < nds * nds; e += blockDim.x) {
      const int r = e / nds, c = e - r * nds;
      sVs[r * lds + c] = Vs[e];
    }
    for (int e = threadIdx.x; e < ndv * ndv; e += blockDim.x) sVv[e] = Vv[e];
    for (int e = threadIdx.x; e < N; e += blockDim.x) {
      sx[e] = 0.0;
      sz[e] = 0.0;
      su[e] = 0.0;
      sq[e] = q[e];
      slam[e] = lam[e];
    }
  }
  for (int e = threadIdx.x; e < ndv * ndv; e += blockDim.x) {
    const int r = e / ndv, c = e - r * ndv;
    sVvT[c * ndv + r] = Vv[e];
  }
  __syncthreads();
  // 16-byte loads of the right operands need an even row stride and aligned rows
  const bool vec_v = (ndv & 1) == 0 && ((reinterpret_cast<uintptr_t>(sVv) | reinterpret_cast<uintptr_t>(sVvT) |
                                        reinterpret_cast<uintptr_t>(srhs) | reinterpret_cast<uintptr_t>(sx) |
                                        reinterpret_cast<uintptr_t>(st1)) & 15) == 0;
  int it = 0;
  for (it = 0; it < 50000; ++it) {
    for (int e = threadIdx.x; e < N; e += blockDim.x)
      srhs[e] = sq[e] + rho * (sz[e] - su[e]) + sigma * sx[e];
    __syncthreads();
    // x = (Vs (x) Vv) diag(lam) (Vs (x) Vv)^T rhs
    cta_gemm24(nds, ndv, nds, sVs, 1, lds, srhs, ndv, st1, ldt, nullptr, vec_v);  // Vs^T R
    __syncthreads();
    cta_gemm24(nds, ndv, ndv, st1, ldt, 1, sVv, ndv, sx, ndv, slam, vec_v);  // ((Vs^T R) Vv) .* lam
    __syncthreads();
    cta_gemm24(nds, ndv, nds, sVs, lds, 1, sx, ndv, st1, ldt, nullptr, vec_v);  // Vs X
    __syncthreads();
    cta_gemm24(nds, ndv, ndv, st1, ldt, 1, sVvT, ndv, sx, ndv, nullptr, vec_v);  // (Vs X) Vv^T
    __syncthreads();
    // Config discretization: over-relaxation x^ = a x + (1 - a) z_old,
    // a = 1.6 (Boyd et al. 2011, sec. 3.4.3; the OSQP default), in the z and
    // u updates; the residuals use the unrelaxed x.  The reference
    // discretization keeps the reference's unrelaxed iteration.
    double nr[5] = {0, 0, 0, 0, 0};
    for (int e = threadIdx.x; e < N; e += blockDim.x) {
      const double xe = sx[e];
      const double zo = sz[e];
      const double xh = d.disc == 1 ? 1.6 * xe + (1.0 - 1.6) * zo : xe;
      double zn = xh + su[e];
      if (zn < 0.0) zn = 0.0;
      sz[e] = zn;
      const double un = su[e] + xh - zn;
      su[e] = un;
      const double pv = xe - zn, dv = rho * (zn - zo);
      nr[0] += pv * pv;
      nr[1] += dv * dv;
      nr[2] += zn * zn;
      nr[3] += xe * xe;
      nr[4] += un * un;
    }
    block_sum<5>(nr, S.red);
    const double eps_p = eps_abs + eps_rel * sqrt(fmax(nr[2], nr[3]));
    const double eps_d = eps_abs + eps_rel * rho * sqrt(nr[4]);
    if (sqrt(nr[0]) < eps_p && sqrt(nr[1]) < eps_d) {
      ++it;
      break;
    }
    // Config discretization: residual balancing of rho (Boyd et al. 2011,
    // sec. 3.4.1) every 10 iterations -- x2 when the primal residual exceeds
    // 10x the dual one, /2 in the opposite case; the scaled dual u is rescaled
    // and the diagonal of the fast diagonalization recomputed.  The reference
    // discretization keeps the reference's fixed rho.
    if (d.disc == 1 && (it + 1) % 10 == 0) {
      const double rp = sqrt(nr[0]), rd = sqrt(nr[1]);
      double f = 1.0;
      if (rp > 10.0 * rd && rho < 1e6) f = 2.0;
      else if (rd > 10.0 * rp && rho > 1e-6) f = 0.5;
      if (f != 1.0) {
        rho *= f;
        const double al = lamreg + sigma + rho;
        for (int e = threadIdx.x; e < N; e += blockDim.x) {
          const int a = e / ndv, b = e - a * ndv;
          const double ls = As[a * nds + a], lv = Av[b * ndv + b];
          slam[e] = 1.0 / ((ls * ls) * (lv * lv) + al);
          su[e] /= f;
        }
        __syncthreads();
      }
    }
  }
  if (sz != z) {
    for (int e = threadIdx.x; e < N; e += blockDim.x) z[e] = sz[e];
    __syncthreads();
  }
  // ---- q0 = max(Dinv c, 0) normalised by m^T q0 ---------------------------
  double* q0 = D + DL.q0;
  const double* ms = D + DL.m_s;
  const double* mv = D + DL.m_v;
  double part = 0.0;
  for (int e = threadIdx.x; e < N; e += blockDim.x) {
    const int a = e / ndv, b = e - a * ndv;
    double v = z[e] / (Ds[a] * Dv[b]);
    if (v < 0.0) v = 0.0;
    q0[e] = v;
    part += (ms[a] * mv[b]) * v;
  }
  const double mq = block_sum1(part, S.red);
  double* y = D + DL.y;
  for (int e = threadIdx.x; e < N; e += blockDim.x) {
    const int a = e / ndv, b = e - a * ndv;
    double v = q0[e];
    if (mq > 0.0) v = v / mq;
    q0[e] = v;
    y[e] = (Ds[a] * Dv[b]) * v;  // scaled state D q0 (solver.mojo:83-86)
  }
  if (threadIdx.x == 0) info[FPE_INFO_ADMM] = it;
}

}  // namespace fpe
