// Device helpers shared by the solve kernels (one CTA of FPE_BLOCK threads per solve).
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "fpe_device.h"

namespace fpe {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic CTA-wide sums of K values; every thread receives the totals.
// red must hold 32*K doubles of shared memory.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) red[k * 32 + wid] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[k * 32 + w];
    v[k] = s;
  }
  __syncthreads();
}

__device__ __forceinline__ double block_sum1(double v, double* red) {
  double a[1] = {v};
  block_sum<1>(a, red);
  return a[0];
}

__device__ __forceinline__ double block_max1(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double m = red[0];
  for (int w = 1; w < nw; ++w) m = fmax(m, red[w]);
  __syncthreads();
  return m;
}

// Block-wide bitonic sort of n doubles in shared memory (buf holds a power of
// two >= n entries; the tail is padded with +inf).
static __device__ void block_sort(double* buf, int n, int cap_pow2) {
  for (int i = n + threadIdx.x; i < cap_pow2; i += blockDim.x) buf[i] = CUDART_INF;
  __syncthreads();
  for (int k = 2; k <= cap_pow2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < cap_pow2; i += blockDim.x) {
        int ixj = i ^ j;
        if (ixj > i) {
          double a = buf[i], b = buf[ixj];
          bool up = (i & k) == 0;
          if ((a > b) == up) {
            buf[i] = b;
            buf[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
  }
}

// Cox-de Boor value of the degree-deg B-spline i on knot vector t (length nt),
// with the half-open degree-0 convention and the last-knot rule of the
// reference (src/numerics/bspline/basis.mojo:25-69).
__device__ __forceinline__ double bs_base(const double* t, int nt, double x, int i) {
  if (i < 0 || i + 1 >= nt) return 0.0;
  double left = t[i], right = t[i + 1], last = t[nt - 1];
  if (left <= x && x < right) return 1.0;
  if (x == last && x == right) return 1.0;
  return 0.0;
}

static __device__ double bs_value(const double* t, int nt, double x, int i, int deg) {
  int nb = nt - deg - 1;
  if (i < 0 || i >= nb) return 0.0;
  double work[4];
  for (int j = 0; j <= deg; ++j) work[j] = bs_base(t, nt, x, i + j);
  for (int k = 1; k <= deg; ++k) {
    int upper = deg - k + 1;
    for (int j = 0; j < upper; ++j) {
      int idx = i + j;
      double d1 = t[idx + k] - t[idx];
      double alpha = d1 != 0.0 ? (x - t[idx]) / d1 : 0.0;
      double d2 = t[idx + k + 1] - t[idx + 1];
      double beta = d2 != 0.0 ? (x - t[idx + 1]) / d2 : 0.0;
      work[j] = alpha * work[j] + (1.0 - beta) * work[j + 1];
    }
  }
  return work[0];
}

// basis.mojo:122-213 (cubic derivative via degree-2 splines).
static __device__ double bs_deriv3(const double* t, int nt, double x, int col) {
  double left = 0.0, right = 0.0;
  double d1 = t[col + 3] - t[col];
  if (d1 != 0.0) left = 3.0 / d1 * bs_value(t, nt, x, col, 2);
  double d2 = t[col + 4] - t[col + 1];
  if (d2 != 0.0) right = 3.0 / d2 * bs_value(t, nt, x, col + 1, 2);
  return left - right;
}

// Recombined cubic basis at x: window of 4 consecutive dofs starting at *c0.
// Recombination (recombination.mojo:14-51): dof c = original B_{c+1}; a
// Neumann end merges B_0 (left) / B_{nb-1} (right) into the adjacent dof, a
// Dirichlet end drops it.  Values with |v| <= 1e-12 are dropped as in
// basis.mojo:85 / :160 before recombination.
static __device__ void recombined_window(const double* t, int nt, double x, bool lneu, bool rneu,
                                  int* c0_out, double* B, double* dB) {
  const int nb = nt - 4;
  const int rc = nb - 2;
  for (int k = 0; k < 4; ++k) B[k] = dB[k] = 0.0;
  // span: largest mu in [3, nb-1] with t[mu] <= x
  int lo = 3, hi = nb - 1;
  if (x < t[0] || x > t[nt - 1]) {
    *c0_out = 0;
    return;
  }
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (t[mid] <= x) lo = mid; else hi = mid - 1;
  }
  int mu = lo;
  int c0 = mu - 4;
  int cmax = rc - 4 > 0 ? rc - 4 : 0;
  if (c0 < 0) c0 = 0;
  if (c0 > cmax) c0 = cmax;
  *c0_out = c0;
  for (int i = mu - 4; i <= mu + 1; ++i) {
    if (i < 0 || i >= nb) continue;
    double v = bs_value(t, nt, x, i, 3);
    double d = bs_deriv3(t, nt, x, i);
    if (!(v > 1e-12 || v < -1e-12)) v = 0.0;
    if (!(d > 1e-12 || d < -1e-12)) d = 0.0;
    if (v == 0.0 && d == 0.0) continue;
    int c;
    if (i == 0) c = (lneu && rc > 0) ? 0 : -1;
    else if (i == nb - 1) c = (rneu && rc > 0) ? rc - 1 : -1;
    else c = i - 1;
    if (c < 0) continue;
    int s = c - c0;
    if (s < 0 || s > 3) continue;
    B[s] += v * 1.0;
    dB[s] += d * 1.0;
  }
}

}  // namespace fpe
