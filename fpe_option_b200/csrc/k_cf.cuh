// Heston characteristic-function prices of European options, FP64.
//
// Heston (1993) writes the call as S0 P1 - K e^{-rT} P2 with
//   P_j = 1/2 + 1/pi  int_0^inf  Re[ e^{-i phi ln K} f_j(phi) / (i phi) ] d phi,
// f_j = exp(C_j + D_j V0 + i phi ln S0).  C_j, D_j are taken in the form of
// Albrecher, Mayer, Schoutens and Tistaert (2007, "The little Heston trap"),
// whose complex logarithm stays on its principal branch:
//   a = rho sigma i phi - b_j,  d = sqrt(a^2 - sigma^2 (2 u_j i phi - phi^2)),
//   m = b_j - rho sigma i phi,  g = (m - d) / (m + d),  e = exp(-d T),
//   C = r i phi T + kappa theta / sigma^2 ((m - d) T - 2 log((1 - g e) / (1 - g))),
//   D = (m - d) / sigma^2 (1 - e) / (1 - g e),
// u_1 = 1/2, b_1 = kappa - rho sigma;  u_2 = -1/2, b_2 = kappa.  Puts follow by
// put-call parity.  The reference engine has no closed-form price; this one
// cross-checks the FPE prices of Europeans (it measures their discretization
// error) and is the fast pricer for European quotes.
//
// Quadrature: composite 16-point Gauss-Legendre on panels of width 1/2 up to
// phi = 50 and 2 beyond, stopped once phi > 40 and a panel adds less than
// 1e-16 (1 + |integral|), or after 4000 panels.  One warp prices one
// (parameter set, strike) pair: lanes 0-15 hold the 16 nodes of P1's panel,
// lanes 16-31 those of P2's, a panel is one integrand evaluation per lane and
// two 16-lane sums; each half stops on its own rule and the warp leaves when
// both have.  The work is FP64 arithmetic and transcendental functions on
// registers (no memory traffic beyond 80 bytes per price).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace fpe {

struct CfNodes {
  double x[16], w[16];  // Gauss-Legendre nodes and weights on [-1, 1]
};

struct Zc {
  double re, im;
};

__device__ __forceinline__ Zc zc(double re, double im = 0.0) { return Zc{re, im}; }
__device__ __forceinline__ Zc operator+(Zc a, Zc b) { return Zc{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Zc operator-(Zc a, Zc b) { return Zc{a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ Zc operator*(Zc a, Zc b) {
  return Zc{fma(a.re, b.re, -a.im * b.im), fma(a.re, b.im, a.im * b.re)};
}
__device__ __forceinline__ Zc operator*(double s, Zc a) { return Zc{s * a.re, s * a.im}; }

// Smith's (1962) division: scale by the larger component of the divisor
// (one ratio and one reciprocal per quotient).
__device__ __forceinline__ Zc operator/(Zc a, Zc b) {
  if (fabs(b.re) >= fabs(b.im)) {
    const double t = b.im / b.re, rd = 1.0 / fma(b.im, t, b.re);
    return Zc{fma(a.im, t, a.re) * rd, fma(-a.re, t, a.im) * rd};
  }
  const double t = b.re / b.im, rd = 1.0 / fma(b.re, t, b.im);
  return Zc{fma(a.re, t, a.im) * rd, fma(a.im, t, -a.re) * rd};
}

// Principal square root (real part >= 0), from |z| without cancellation.
__device__ __forceinline__ Zc zsqrt(Zc z) {
  const double m = hypot(z.re, z.im);
  if (m == 0.0) return Zc{0.0, z.im};
  if (z.re >= 0.0) {
    const double t = sqrt(0.5 * (m + z.re));
    return Zc{t, z.im / (2.0 * t)};
  }
  const double t = sqrt(0.5 * (m - z.re));
  return Zc{fabs(z.im) / (2.0 * t), copysign(t, z.im)};
}

__device__ __forceinline__ Zc zexp(Zc z) {
  double s, c;
  sincos(z.im, &s, &c);
  const double e = exp(z.re);
  return Zc{e * c, e * s};
}

// Principal logarithm.
__device__ __forceinline__ Zc zlog(Zc z) { return Zc{log(hypot(z.re, z.im)), atan2(z.im, z.re)}; }

struct CfModel {
  double kappa, theta, sigma, rho, r, T, lnS, lnK, V0;
};

// Re[e^{-i phi ln K} f_j(phi) / (i phi)] for j = 1 (P1) or 2 (P2).
__device__ __forceinline__ double cf_integrand(const CfModel& m, double phi, int j) {
  const double u = j == 1 ? 0.5 : -0.5;
  const double b = j == 1 ? m.kappa - m.rho * m.sigma : m.kappa;
  const double s2 = m.sigma * m.sigma, rsp = m.rho * m.sigma * phi;
  const Zc a = zc(-b, rsp);
  const Zc d = zsqrt(a * a - s2 * zc(-phi * phi, 2.0 * u * phi));
  const Zc mm = zc(b, -rsp);
  const Zc md = mm - d;
  const Zc g = md / (mm + d);
  const Zc e = zexp(-m.T * d);
  const Zc one = zc(1.0);
  const Zc ge1 = one - g * e;
  const Zc C = zc(0.0, m.r * phi * m.T) +
               (m.kappa * m.theta / s2) * (m.T * md - 2.0 * zlog(ge1 / (one - g)));
  const Zc D = (1.0 / s2) * (md * ((one - e) / ge1));
  // e^{-i phi ln K} f = exp(C + D V0 + i phi (ln S0 - ln K)); divided by i phi
  // its real part is Im(.) / phi.
  const Zc f = zexp(C + m.V0 * D + zc(0.0, phi * (m.lnS - m.lnK)));
  return f.im / phi;
}

constexpr int kCfPanels = 4000;
constexpr int kCfWarps = 4;  // prices per 128-thread block

// params: n rows of (kappa, theta, sigma, rho, r, T, S0, V0); put may be null.
// Rows outside the model's domain (kappa, theta, sigma, T, S0, K <= 0, V0 < 0,
// |rho| > 1 or any non-finite entry) give NaN.
__global__ void __launch_bounds__(32 * kCfWarps) k_heston_cf(const double* __restrict__ params,
                                                            const double* __restrict__ strikes,
                                                            const int32_t* __restrict__ put, int32_t n,
                                                            CfNodes q, double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const long long item = (long long)blockIdx.x * kCfWarps + (threadIdx.x >> 5);
  if (item >= n) return;
  const double* p = params + item * 8;
  const double kappa = p[0], theta = p[1], sigma = p[2], rho = p[3], r = p[4], T = p[5], S0 = p[6],
               V0 = p[7], K = strikes[item];
  const bool ok = kappa > 0.0 && theta > 0.0 && sigma > 0.0 && T > 0.0 && S0 > 0.0 && K > 0.0 &&
                  V0 >= 0.0 && rho >= -1.0 && rho <= 1.0 && isfinite(kappa) && isfinite(theta) &&
                  isfinite(sigma) && isfinite(r) && isfinite(T) && isfinite(S0) && isfinite(V0) &&
                  isfinite(K);
  if (!ok) {
    if (lane == 0) out[item] = __longlong_as_double(0x7ff8000000000000ll);
    return;
  }
  const CfModel m{kappa, theta, sigma, rho, r, T, log(S0), log(K), V0};
  const int j = 1 + (lane >> 4);
  const double x = q.x[lane & 15], w = q.w[lane & 15];
  double acc = 0.0, lo = 0.0;
  bool done = false;
  for (int seg = 0; seg < kCfPanels; ++seg) {
    const double width = lo < 50.0 ? 0.5 : 2.0;
    const double hi = lo + width, mid = 0.5 * (lo + hi), half = 0.5 * width;
    double v = done ? 0.0 : w * cf_integrand(m, mid + half * x, j);
#pragma unroll
    for (int o = 8; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const double part = v * half;
    if (!done) {
      acc += part;
      if (hi > 40.0 && fabs(part) < 1e-16 * (1.0 + fabs(acc))) done = true;
    }
    lo = hi;
    if (__all_sync(0xffffffffu, done)) break;
  }
  const double P = 0.5 + acc / 3.14159265358979323846;
  const double P2 = __shfl_sync(0xffffffffu, P, 16);
  if (lane == 0) {
    const double disc = K * exp(-r * T);
    const double call = S0 * P - disc * P2;
    out[item] = (put && put[item]) ? call - S0 + disc : call;
  }
}

}  // namespace fpe
