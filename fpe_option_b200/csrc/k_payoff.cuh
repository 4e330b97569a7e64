// Terminal-density payoff integration and the full-grid PDF, FP64.
//
// Reference: _price_at (src/server/pricer.mojo:27-64) evaluates
//   price_k = e^{-rT} sum_i payoff_k(s_i) sw_i sum_j vw_j pdf_ij,
//   pdf = (Bs (x) Bv) q_T on the quadrature grid (pdf.mojo:28-32),
// with BarrierPayoff activity rules (payoffs.mojo:19-50).  The same sum in
// reduced form needs no 2-D grid:
//   r_a = sum_b q_ab mv_b,  mv_b = sum_j Bv_jb vw_j,
//   price_k = e^{-rT} sum_i payoff_k(s_i) sw_i sum_a Bs_ia r_a.
// The config discretization integrates the payoff exactly instead: knot spans
// are split at the strike and 4-point Gauss-Legendre is exact on each piece.
#pragma once
#include "dev_common.cuh"

namespace fpe {

__device__ __forceinline__ double payoff_value(int type, double S, double K, double B) {
  bool active;
  if (type == 0 || type == 1) active = S <= B;
  else if (type == 2 || type == 3) active = S > B;
  else if (type == 4 || type == 5) active = S >= B;
  else if (type == 6 || type == 7) active = S < B;
  else active = true;
  if (!active) return 0.0;
  double v = (type % 2 == 0) ? S - K : K - S;
  return v > 0.0 ? v : 0.0;
}

struct PayoffSmem {
  double red[32 * 2];
  double r[FPE_MAX_NDOF_S];
  double mvo[FPE_MAX_NDOF_V];  // v weights of the calibration-objective rule
};

__global__ void __launch_bounds__(FPE_BLOCK) k_payoff(const FpeSolveDesc* __restrict__ descs,
                                                      double* __restrict__ darena,
                                                      int32_t* __restrict__ iarena,
                                                      int32_t* __restrict__ infos,
                                                      const double* __restrict__ strikes,
                                                      double* __restrict__ prices) {
  __shared__ PayoffSmem S;
  const FpeSolveDesc d = descs[blockIdx.x];
  const FpeDLayout DL = fpe_dlayout(d);
  const FpeILayout IL = fpe_ilayout(d);
  double* D = darena + d.off_d;
  int32_t* I = iarena + d.off_i;
  const int32_t* info = infos + size_t(blockIdx.x) * FPE_INFO_COUNT;
  const int nk = d.n_strikes;
  if (info[FPE_INFO_STATUS] != 0 && info[FPE_INFO_STATUS] != FPE_ERR_MAX_STEPS &&
      info[FPE_INFO_STATUS] != FPE_ERR_STEP_UNDERFLOW) {
    for (int k = threadIdx.x; k < nk; k += blockDim.x) prices[d.strike_off + k] = CUDART_NAN;
    return;
  }
  const int nds = info[FPE_INFO_NDOF_S], ndv = info[FPE_INFO_NDOF_V];
  const double* qT = D + DL.qT;
  const double* mv = D + DL.m_v;
  // The calibration objective (objective.mojo:26-50) sums payoff * pdf * ds * dv
  // over the quadrature points with half the neighbour spacing as weight (1 at
  // both ends) and no discount.  In reduced form its v weights are
  // mv'_b = sum_q Bv_qb dv_q, and ds replaces the s quadrature weight below.
  const bool objective = d.disc == 0 && d.price_rule == 1;
  if (objective) {
    const int nqv = info[FPE_INFO_NQ_V];
    const double* vp = D + DL.qp_v;
    const double* Bv = D + DL.B_v;
    const int32_t* c0v = I + IL.c0_v;
    for (int b = threadIdx.x; b < ndv; b += blockDim.x) {
      double acc = 0.0;
      for (int q = 0; q < nqv; ++q) {
        const int t = b - c0v[q];
        if (t < 0 || t > 3) continue;
        const double dv = (q > 0 && q < nqv - 1) ? 0.5 * (vp[q + 1] - vp[q - 1]) : 1.0;
        acc += Bv[4 * q + t] * dv;
      }
      S.mvo[b] = acc;
    }
    __syncthreads();
    mv = S.mvo;
  }
  for (int a = threadIdx.x; a < nds; a += blockDim.x) {
    double acc = 0.0;
    for (int b = 0; b < ndv; ++b) acc += qT[a * ndv + b] * mv[b];
    S.r[a] = acc;
  }
  __syncthreads();
  const double disc = objective ? 1.0 : exp(-d.r * d.T);
  const double* ks = strikes + d.strike_off;
  if (d.disc == 0) {
    const int nq = info[FPE_INFO_NQ_S];
    const double* qw = D + DL.qw_s;
    const double* qp = D + DL.qp_s;
    const double* Bt = D + DL.B_s;
    const int32_t* c0 = I + IL.c0_s;
    for (int k = 0; k < nk; ++k) {
      const double K = ks[k];
      double part = 0.0;
      for (int p = threadIdx.x; p < nq; p += blockDim.x) {
        const double pay = payoff_value(d.type, qp[p], K, d.barrier);
        if (pay == 0.0) continue;
        const int cc = c0[p];
        double dot = 0.0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          const int a = cc + s;
          if (a < nds) dot += Bt[4 * p + s] * S.r[a];
        }
        const double wp = objective ? ((p > 0 && p < nq - 1) ? 0.5 * (qp[p + 1] - qp[p - 1]) : 1.0) : qw[p];
        part += pay * (dot * wp);
      }
      const double tot = block_sum1(part, S.red);
      if (threadIdx.x == 0) prices[d.strike_off + k] = tot * disc;
    }
  } else {
    const int nkn = info[FPE_INFO_NKNOT_S];
    const double* kn = D + DL.knot_s;
    const double J = d.smax - d.smin;
    const bool lneu = d.left_neu != 0, rneu = d.right_neu != 0;
    double glx[4], glw[4];
    {
      double a = sqrt(3.0 / 7.0 - 2.0 / 7.0 * sqrt(6.0 / 5.0));
      double b = sqrt(3.0 / 7.0 + 2.0 / 7.0 * sqrt(6.0 / 5.0));
      double wa = (18.0 + sqrt(30.0)) / 36.0, wb = (18.0 - sqrt(30.0)) / 36.0;
      glx[0] = -b; glx[1] = -a; glx[2] = a; glx[3] = b;
      glw[0] = wb; glw[1] = wa; glw[2] = wa; glw[3] = wb;
    }
    const int nspan = nkn - 1;
    for (int k = 0; k < nk; ++k) {
      const double K = ks[k];
      const double kx = (K - d.smin) / J;
      double part = 0.0;
      for (int e = threadIdx.x; e < nspan * 2 * 4; e += blockDim.x) {
        const int sp = e >> 3, piece = (e >> 2) & 1, g = e & 3;
        const double a = kn[sp], b = kn[sp + 1];
        if (!(b > a)) continue;
        double lo = a, hi = b;
        if (kx > a && kx < b) {
          if (piece == 0) hi = kx; else lo = kx;
        } else if (piece == 1) {
          continue;
        }
        const double mid = 0.5 * (lo + hi), hw = 0.5 * (hi - lo);
        const double x = mid + hw * glx[g];
        const double Sx = d.smin + x * J;
        const double pay = payoff_value(d.type, Sx, K, d.barrier);
        if (pay == 0.0) continue;
        int c0;
        double Bw[4], dBw[4];
        recombined_window(kn, nkn, x, lneu, rneu, &c0, Bw, dBw);
        double dot = 0.0;
        for (int s = 0; s < 4; ++s)
          if (c0 + s < nds) dot += Bw[s] * S.r[c0 + s];
        part += pay * dot * (hw * glw[g] * J);
      }
      const double tot = block_sum1(part, S.red);
      if (threadIdx.x == 0) prices[d.strike_off + k] = tot * disc;
    }
  }
}

// pdf[p][q] = sum_a sum_b Bs(p, a) Bv(q, b) qT[a, b] on the quadrature grid.
__global__ void k_pdf(const FpeSolveDesc* __restrict__ descs, const double* __restrict__ darena,
                      const int32_t* __restrict__ iarena, const int32_t* __restrict__ infos,
                      int solve, double* __restrict__ out) {
  const FpeSolveDesc d = descs[solve];
  const FpeDLayout DL = fpe_dlayout(d);
  const FpeILayout IL = fpe_ilayout(d);
  const double* D = darena + d.off_d;
  const int32_t* I = iarena + d.off_i;
  const int32_t* info = infos + size_t(solve) * FPE_INFO_COUNT;
  const int nqs = info[FPE_INFO_NQ_S], nqv = info[FPE_INFO_NQ_V];
  const int nds = info[FPE_INFO_NDOF_S], ndv = info[FPE_INFO_NDOF_V];
  const double* qT = D + DL.qT;
  const double* Bs = D + DL.B_s;
  const double* Bv = D + DL.B_v;
  const int32_t* c0s = I + IL.c0_s;
  const int32_t* c0v = I + IL.c0_v;
  const size_t total = size_t(nqs) * nqv;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < total;
       e += size_t(gridDim.x) * blockDim.x) {
    const int p = int(e / nqv), q = int(e - size_t(p) * nqv);
    const int cs = c0s[p], cv = c0v[q];
    double acc = 0.0;
    for (int s = 0; s < 4; ++s) {
      const int a = cs + s;
      if (a >= nds) continue;
      const double bs = Bs[4 * p + s];
      if (bs == 0.0) continue;
      double inner = 0.0;
      for (int t = 0; t < 4; ++t) {
        const int b = cv + t;
        if (b < ndv) inner += Bv[4 * q + t] * qT[a * ndv + b];
      }
      acc += bs * inner;
    }
    out[e] = acc;
  }
}

}  // namespace fpe
