// Galerkin 1-D factor assembly by Gauss-Legendre quadrature and the D-scaled
// Kronecker operator factors, one CTA per solve.
//
// Reference: mass_from_cached / stiffness_from_cached
// (src/engines/fpe/galerkin.mojo:16-125) build M = Ns (x) Nv and
//   K = S1s(x)V1v + S2s(x)V2v + Ns(x)(k5 V4 + k6 V5) + S4s(x)V2v
//     + k8 Ns(x)V6 + (S3s(x)V3v)^T + S3s(x)V3v
// with S1s = k1 Ss, S2s = k2 Ss, S3s = k4 Ss, S4s = k3 Tss.  Regrouped here
// into four Kronecker terms of banded (7-diagonal) 1-D factors:
//   K = Ss(x)B1 + Tss(x)B2 + Ns(x)B3 + Ss^T(x)B4
//   B1 = k1 Nv + k2 V2 + k4 V3, B2 = k3 V2, B3 = k5 V4 + k6 V5 + k8 V6, B4 = k4 V3^T
// and scaled by D = sqrt(diag M) = Ds (x) Dv (solver.mojo:57-87).
#pragma once
#include "dev_common.cuh"

namespace fpe {

// One warp per dof row.  Lanes stride over the quadrature nodes in the row's
// support; each lane keeps 7 band sums per factor; shuffle reduction at the end.
template <int NF>
__device__ void galerkin_axis(int ndof, const double* __restrict__ qw, const double* __restrict__ qp,
                              const double* __restrict__ Bt, const double* __restrict__ dBt,
                              const int32_t* __restrict__ c0t, const int32_t* __restrict__ rng,
                              double* __restrict__ fac, double* __restrict__ msum, bool is_v) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int i = wid; i < ndof; i += nw) {
    double acc[NF][7];
    double macc = 0.0;
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int dd = 0; dd < 7; ++dd) acc[f][dd] = 0.0;
    const int q0 = rng[2 * i], q1 = rng[2 * i + 1];
    for (int q = q0 + lane; q < q1; q += 32) {
      const int c0 = c0t[q];
      const int li = i - c0;
      if (li < 0 || li > 3) continue;
      const double w = qw[q];
      if (w == 0.0) continue;
      const double x = qp[q];
      double Bw[4], dBw[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        Bw[k] = Bt[4 * q + k];
        dBw[k] = dBt[4 * q + k];
      }
      const double Li = Bw[li], dLi = dBw[li];
      macc += Li * w;
#pragma unroll
      for (int dd = 0; dd < 7; ++dd) {
        const int lj = li + dd - 3;
        if (lj < 0 || lj > 3) continue;
        const double Rj = Bw[lj], dRj = dBw[lj];
        if (!is_v) {
          // 0 Ns: B,B,w   1 Ss: dB,B,s w   2 Tss: dB,dB,s^2 w
          acc[0][dd] += Li * (w * Rj);
          if (NF > 1) acc[1 % NF][dd] += dLi * ((x * w) * Rj);
          if (NF > 2) acc[2 % NF][dd] += dLi * ((x * x * w) * dRj);
        } else {
          // 0 Nv: B,B,w  1 V2: B,B,v w  2 V3: B,dB,v w  3 V4: dB,B,w  4 V5: dB,B,v w  5 V6: dB,dB,v w
          const double vw = x * w;
          acc[0][dd] += Li * (w * Rj);
          if (NF > 5) {
            acc[1][dd] += Li * (vw * Rj);
            acc[2][dd] += Li * (vw * dRj);
            acc[3][dd] += dLi * (w * Rj);
            acc[4][dd] += dLi * (vw * Rj);
            acc[5][dd] += dLi * (vw * dRj);
          }
        }
      }
    }
    macc = warp_sum(macc);
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int dd = 0; dd < 7; ++dd) acc[f][dd] = warp_sum(acc[f][dd]);
    if (lane == 0) {
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int dd = 0; dd < 7; ++dd) {
          const int j = i + dd - 3;
          fac[(size_t(f) * ndof + i) * 7 + dd] = (j >= 0 && j < ndof) ? acc[f][dd] : 0.0;
        }
      msum[i] = macc;
    }
  }
}

__global__ void __launch_bounds__(FPE_BLOCK) k_galerkin(const FpeSolveDesc* __restrict__ descs,
                                                        double* __restrict__ darena,
                                                        int32_t* __restrict__ iarena, int32_t* __restrict__ infos) {
  const FpeSolveDesc d = descs[blockIdx.x];
  const FpeDLayout DL = fpe_dlayout(d);
  const FpeILayout IL = fpe_ilayout(d);
  double* D = darena + d.off_d;
  int32_t* I = iarena + d.off_i;
  const int32_t* info = infos + size_t(blockIdx.x) * FPE_INFO_COUNT;
  if (info[FPE_INFO_STATUS] != 0) return;
  const int nds = info[FPE_INFO_NDOF_S], ndv = info[FPE_INFO_NDOF_V];
  double* fs = D + DL.fac_s;
  double* fv = D + DL.fac_v;
  galerkin_axis<FPE_NFAC_S>(nds, D + DL.qw_s, D + DL.qp_s, D + DL.B_s, D + DL.dB_s, I + IL.c0_s,
                            I + IL.rng_s, fs, D + DL.m_s, false);
  galerkin_axis<FPE_NFAC_V>(ndv, D + DL.qw_v, D + DL.qp_v, D + DL.B_v, D + DL.dB_v, I + IL.c0_v,
                            I + IL.rng_v, fv, D + DL.m_v, true);
  __syncthreads();

  // D-scaling and the operator factors (galerkin.mojo:68-74 constants).
  const double J = d.smax - d.smin;
  const double k1 = (-d.r + 0.5 * d.rho * d.sigma) / J;
  const double k2 = 1.0 / J;
  const double k3 = 0.5 / (J * J);
  const double k4 = 0.5 * d.rho * d.sigma / J;
  const double k5 = 0.5 * d.sigma * d.sigma - d.kappa * d.theta;
  const double k6 = d.kappa + 0.5 * d.rho * d.sigma;
  const double k8 = 0.5 * d.sigma * d.sigma;
  double* Ds = D + DL.D_s;
  double* Dv = D + DL.D_v;
  for (int i = threadIdx.x; i < nds; i += blockDim.x) {
    double m = fs[i * 7 + 3];
    Ds[i] = m > 1e-30 ? sqrt(m) : 1.0;
  }
  for (int j = threadIdx.x; j < ndv; j += blockDim.x) {
    double m = fv[j * 7 + 3];
    Dv[j] = m > 1e-30 ? sqrt(m) : 1.0;
  }
  __syncthreads();
  double* os = D + DL.op_s;
  double* ov = D + DL.op_v;
  auto FS = [&](int f, int i, int dd) { return fs[(size_t(f) * nds + i) * 7 + dd]; };
  auto FV = [&](int f, int j, int dd) { return fv[(size_t(f) * ndv + j) * 7 + dd]; };
  for (int e = threadIdx.x; e < nds * 7; e += blockDim.x) {
    const int i = e / 7, dd = e % 7, k = i + dd - 3;
    double a = 0, b = 0, c = 0, t = 0;
    if (k >= 0 && k < nds) {
      const double sc = 1.0 / (Ds[i] * Ds[k]);
      a = FS(0, i, dd) * sc;
      b = FS(1, i, dd) * sc;
      c = FS(2, i, dd) * sc;
      t = FS(1, k, 6 - dd) * sc;  // (Ss^T)[i][k] = Ss[k][i]
    }
    os[(0 * nds + i) * 7 + dd] = a;
    os[(1 * nds + i) * 7 + dd] = b;
    os[(2 * nds + i) * 7 + dd] = c;
    os[(3 * nds + i) * 7 + dd] = t;
  }
  for (int e = threadIdx.x; e < ndv * 7; e += blockDim.x) {
    const int j = e / 7, dd = e % 7, l = j + dd - 3;
    double av = 0, b1 = 0, b2 = 0, b3 = 0, b4 = 0;
    if (l >= 0 && l < ndv) {
      const double sc = 1.0 / (Dv[j] * Dv[l]);
      av = FV(0, j, dd) * sc;
      b1 = (k1 * FV(0, j, dd) + k2 * FV(1, j, dd) + k4 * FV(2, j, dd)) * sc;
      b2 = (k3 * FV(1, j, dd)) * sc;
      b3 = (k5 * FV(3, j, dd) + k6 * FV(4, j, dd) + k8 * FV(5, j, dd)) * sc;
      b4 = (k4 * FV(2, l, 6 - dd)) * sc;  // (V3^T)[j][l] = V3[l][j]
    }
    ov[(0 * ndv + j) * 7 + dd] = av;
    ov[(1 * ndv + j) * 7 + dd] = b1;
    ov[(2 * ndv + j) * 7 + dd] = b2;
    ov[(3 * ndv + j) * 7 + dd] = b3;
    ov[(4 * ndv + j) * 7 + dd] = b4;
  }
}

}  // namespace fpe
