// Interpolation of a terminal density tabulated on a tensor grid, FP64
// (reference src/server/interpolator.mojo:14-198): Catmull-Rom bicubic on the
// 4 x 4 neighbourhood of the cell holding (s, v), indices clamped at the
// edges, the local coordinates t in [0, 1] clamped; bilinear when either axis
// has fewer than 4 points.  One thread per query point; the grid is read
// through L1/L2 (a few MB, shared by all queries).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace fpe {

// Cell index i with p[i] <= x < p[i+1] (interpolator.mojo:44-60): 0 for
// x <= p[0], n - 2 for x >= p[n-1] and for a NaN x.  Binary search over the
// nondecreasing points returns the same cell as the reference's linear scan:
// only one cell satisfies p[i] <= x < p[i+1].
__device__ __forceinline__ int interp_cell(const double* p, int n, double x) {
  if (n <= 1) return 0;
  if (x <= p[0]) return 0;
  if (!(x < p[n - 1])) return n - 2;
  int lo = 0, hi = n - 1;  // p[lo] <= x < p[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (p[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Catmull-Rom weights at t (interpolator.mojo:13-30).
__device__ __forceinline__ void catmull_rom(double t, double (&w)[4]) {
  const double t2 = t * t, t3 = t2 * t;
  w[0] = -0.5 * t3 + t2 - 0.5 * t;
  w[1] = 1.5 * t3 - 2.5 * t2 + 1.0;
  w[2] = -1.5 * t3 + 2.0 * t2 + 0.5 * t;
  w[3] = 0.5 * t3 - 0.5 * t2;
}

__device__ __forceinline__ double interp_local(const double* p, int i, double x) {
  double t = 0.0;
  if (p[i + 1] > p[i]) t = (x - p[i]) / (p[i + 1] - p[i]);
  return t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
}

// pdf row-major n_s x n_v; out[k] = pdf interpolated at (s[k], v[k]).
__global__ void k_pdf_interp(const double* __restrict__ sp, int n_s, const double* __restrict__ vp, int n_v,
                             const double* __restrict__ pdf, const double* __restrict__ s,
                             const double* __restrict__ v, int n, double* __restrict__ out) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double x = s[k], y = v[k];
  const int i = interp_cell(sp, n_s, x), j = interp_cell(vp, n_v, y);
  const double ts = interp_local(sp, i, x), tv = interp_local(vp, j, y);
  if (n_s >= 4 && n_v >= 4) {
    double ws[4], wv[4];
    catmull_rom(ts, ws);
    catmull_rom(tv, wv);
    double acc = 0.0;
#pragma unroll
    for (int di = 0; di < 4; ++di) {
      const int ii = min(max(i - 1 + di, 0), n_s - 1);
      const double* row = pdf + size_t(ii) * n_v;
#pragma unroll
      for (int dj = 0; dj < 4; ++dj) {
        const int jj = min(max(j - 1 + dj, 0), n_v - 1);
        acc += ws[di] * wv[dj] * row[jj];
      }
    }
    out[k] = acc;
  } else {
    const double f00 = pdf[size_t(i) * n_v + j], f10 = pdf[size_t(i + 1) * n_v + j];
    const double f01 = pdf[size_t(i) * n_v + j + 1], f11 = pdf[size_t(i + 1) * n_v + j + 1];
    out[k] = (1.0 - ts) * (1.0 - tv) * f00 + ts * (1.0 - tv) * f10 + (1.0 - ts) * tv * f01 + ts * tv * f11;
  }
}

}  // namespace fpe
