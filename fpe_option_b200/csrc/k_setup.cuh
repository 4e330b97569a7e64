// Discretization on the device: knot vectors, quadrature grids and the
// recombined basis tables at the quadrature nodes, one CTA per solve.
//
// Reference rules: GenerateKnots (src/numerics/bspline/knots.mojo:101-270),
// _grid_create / _compute_quad_points / _compute_quad_weights
// (src/engines/fpe/domain.mojo:20-111), FPEDomain (domain.mojo:169-237).
// Config rules: sinh-stretched clamped knots and textbook 4-point
// Gauss-Legendre per knot span.
#pragma once
#include "dev_common.cuh"

namespace fpe {

__device__ __forceinline__ void d_linspace(double* out, int& n, double a, double b, int cnt) {
  if (cnt <= 0) return;
  if (cnt == 1) {
    out[n++] = a;
    return;
  }
  double step = (b - a) / double(cnt - 1);
  for (int i = 0; i < cnt; ++i) out[n++] = a + double(i) * step;
}

__device__ void insertion_sort(double* a, int n) {
  for (int i = 1; i < n; ++i) {
    double v = a[i];
    int j = i - 1;
    while (j >= 0 && a[j] > v) {
      a[j + 1] = a[j];
      --j;
    }
    a[j + 1] = v;
  }
}

__device__ __forceinline__ double py_fmod(double a, double b) {
  double r = fmod(a, b);
  if (r != 0.0 && ((r < 0.0) != (b < 0.0))) r += b;
  return r;
}

// GenerateKnots.generate_knots(method="non-uniform", degree=3, cheby_num=13)
// executed by one thread; scratch holds >= 4*n + 64 doubles.  Returns the
// knot count (or -1 when cap is exceeded).
__device__ int gen_knots_reference(double* out, int cap, int n, double center, double b0,
                                   double b1, double mean, double sd, double* scratch) {
  const int p = 3;
  double bn0 = 0.0, bn1 = 0.0;  // normalize([b0, b1])
  {
    double mn = fmin(b0, b1), mx = fmax(b0, b1), range = mx - mn;
    if (range != 0.0) {
      double inv = 1.0 / range;
      bn0 = (b0 - mn) * inv;
      bn1 = (b1 - mn) * inv;
    }
  }
  double x_min = mean - 4.5 * sd, x_max = mean + 4.5 * sd;
  double x_min_n = (x_min - b0) / (b1 - b0), x_max_n = (x_max - b0) / (b1 - b0);
  int internal_num = n - 2 * p;
  // chebyshev_knots(13, x_min, x_max), normalized and sorted (knots.mojo:165-188)
  double* xn = scratch;  // 15
  {
    const int nc = 13;
    double scale = (x_max - x_min) / 2.0, shift = (x_min + x_max) / 2.0;
    double inv_2n = CUDART_PI / (2.0 * double(nc));
    double tmp[15];
    tmp[0] = x_min;
    tmp[14] = x_max;
    for (int i = 0; i < nc; ++i) tmp[1 + i] = scale * cos((2.0 * double(i) + 1.0) * inv_2n) + shift;
    for (int i = 0; i < 15; ++i) xn[i] = (tmp[i] - b0) / (b1 - b0);
    insertion_sort(xn, 15);
  }
  // func_parabolic(internal_num, (bn0, bn1)) (knots.mojo:101-163)
  double* y = scratch + 16;
  int ny = 0;
  {
    double c = center, low = bn0, high = bn1;
    double divide = sqrt((high - c) / (c - low)) + 1.0;
    int n_adj;
    if (py_fmod(double(internal_num), divide) == 0.0)
      n_adj = internal_num;
    else
      n_adj = int(double(internal_num) / divide) * int(divide);
    if (n_adj < 1) n_adj = internal_num;
    double factor = 2.0;
    double a = fabs(2.0 * (low - c) / (factor * factor));
    double upward = sqrt(2.0 * (high - c) / a) + factor;
    double* x = y + (n + 16);
    int nx = 0;
    d_linspace(x, nx, 0.0, upward, n_adj - 1);
    x[nx++] = factor;
    insertion_sort(x, nx);
    for (int i = 0; i < nx; ++i) y[i] = -0.5 * a * (x[i] - factor) * (x[i] - factor) + c;
    double min_dist = fabs(y[0] - c);
    int ci = 0;
    for (int i = 1; i < nx; ++i) {
      double d = fabs(y[i] - c);
      if (d < min_dist) {
        min_dist = d;
        ci = i;
      }
    }
    for (int i = ci + 1; i < nx; ++i) y[i] = 0.5 * a * (x[i] - factor) * (x[i] - factor) + c;
    insertion_sort(y, nx);
    ny = nx;
  }
  // merge left + chebyshev + right, sort, round to 1e-8, dedup (knots.mojo:224-251)
  double* merged = y + 2 * (n + 16);
  int nm = 0;
  for (int i = 0; i < ny; ++i)
    if (fabs(y[i] - x_min_n) < 1e-10 || y[i] < x_min_n) merged[nm++] = y[i];
  for (int i = 0; i < 15; ++i) merged[nm++] = xn[i];
  for (int i = 0; i < ny; ++i)
    if (fabs(y[i] - x_max_n) < 1e-10 || y[i] > x_max_n) merged[nm++] = y[i];
  insertion_sort(merged, nm);
  for (int i = 0; i < nm; ++i) merged[i] = round(merged[i] * 1e8) / 1e8;
  int il = 0;
  double* internal = merged;  // dedup in place
  for (int i = 0; i < nm; ++i) {
    if (il == 0 || merged[i] > internal[il - 1] + 1e-9) internal[il++] = merged[i];
  }
  int total = 2 * p + il;
  if (total > cap) return -1;
  // internal[] aliases merged[]; copy after the padding is placed safely
  for (int i = il - 1; i >= 0; --i) out[p + i] = internal[i];
  for (int i = 0; i < p; ++i) out[i] = bn0;
  for (int i = p + il; i < total; ++i) out[i] = bn1;
  return total;
}

// Config knots: sinh-stretched distinct knots on [lo, hi] clustered at
// center with scale c, mapped to [0, 1] when normalize is set, padded with
// three repeats of each end (clamped, multiplicity 4).
__device__ int gen_knots_config(double* out, int cap, int n, double lo, double hi, double center,
                                double c, bool normalize_to_unit) {
  if (n + 6 > cap || n < 2) return -1;
  double a0 = asinh((lo - center) / c), a1 = asinh((hi - center) / c);
  for (int j = 0; j < n; ++j) {
    double a = a0 + (a1 - a0) * double(j) / double(n - 1);
    double k = center + c * sinh(a);
    if (j == 0) k = lo;
    if (j == n - 1) k = hi;
    if (normalize_to_unit) k = (k - lo) / (hi - lo);
    out[3 + j] = k;
  }
  if (normalize_to_unit) {
    out[3] = 0.0;
    out[3 + n - 1] = 1.0;
  }
  for (int i = 0; i < 3; ++i) {
    out[i] = out[3];
    out[n + 3 + i] = out[n + 2];
  }
  return n + 6;
}

// Reference quadrature grid before dedup (domain.mojo:20-66).
__device__ int grid_reference_raw(double* g, double center, double sd, double lo, double hi,
                                  int num_insert, bool is_v) {
  int n = 0;
  double lb = center - 5.0 * sd, ub = center + 5.0 * sd;
  int left_trail = int(double(num_insert) * 0.2);
  int num_interm = int(double(num_insert) * 0.3);
  int right_trail = int(double(num_insert) * 0.5);
  if (left_trail < 1) left_trail = 1;
  if (num_interm < 3) num_interm = 3;
  if (right_trail < 1) right_trail = 1;
  int i3 = num_interm / 3;
  d_linspace(g, n, lo, lb, left_trail);
  d_linspace(g, n, lb, center - sd / 5.0, i3 > 1 ? i3 : 1);
  d_linspace(g, n, center - sd / 5.0, center + sd / 5.0, i3 > 2 ? i3 : 2);
  g[n++] = center;
  d_linspace(g, n, center + sd / 5.0, ub, i3 > 1 ? i3 : 1);
  d_linspace(g, n, ub, hi, right_trail);
  int tail = int(double(num_insert) * 0.1);
  d_linspace(g, n, hi - 0.1, hi, tail > 2 ? tail : 2);
  if (is_v) {
    int vz = int(double(num_insert) * 0.2);
    d_linspace(g, n, 0.0, 0.01, vz > 2 ? vz : 2);
  }
  return n;
}

struct SetupSmem {
  double knots[2][512];
  double sortbuf[8192];
  double scratch[2048];
  int cnt[8];
};

// Quadrature rule on [-1, 1]: the reference's order-4 rule keeps the node
// formula sqrt(3/7 -+ 2/7 sqrt(5/6)) of knots.mojo:33-39 (not the textbook
// sqrt(6/5)); the config discretization uses the textbook rule.
__device__ __forceinline__ void gl4(bool reference, double* x, double* w) {
  if (reference) {
    double s1 = sqrt(3.0 / 7.0 + 2.0 / 7.0 * sqrt(5.0 / 6.0));
    double s2 = sqrt(3.0 / 7.0 - 2.0 / 7.0 * sqrt(5.0 / 6.0));
    double w1 = (18.0 - sqrt(30.0)) / 36.0, w2 = (18.0 + sqrt(30.0)) / 36.0;
    x[0] = -s1; x[1] = -s2; x[2] = s2; x[3] = s1;
    w[0] = w1; w[1] = w2; w[2] = w2; w[3] = w1;
  } else {
    double a = sqrt(3.0 / 7.0 - 2.0 / 7.0 * sqrt(6.0 / 5.0));
    double b = sqrt(3.0 / 7.0 + 2.0 / 7.0 * sqrt(6.0 / 5.0));
    double wa = (18.0 + sqrt(30.0)) / 36.0, wb = (18.0 - sqrt(30.0)) / 36.0;
    x[0] = -b; x[1] = -a; x[2] = a; x[3] = b;
    w[0] = wb; w[1] = wa; w[2] = wa; w[3] = wb;
  }
}

__global__ void __launch_bounds__(FPE_BLOCK) k_setup(const FpeSolveDesc* __restrict__ descs,
                                                     double* __restrict__ darena,
                                                     int32_t* __restrict__ iarena, int32_t* __restrict__ infos) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SetupSmem& S = *reinterpret_cast<SetupSmem*>(smem_raw);
  const FpeSolveDesc d = descs[blockIdx.x];
  const FpeDLayout DL = fpe_dlayout(d);
  const FpeILayout IL = fpe_ilayout(d);
  double* D = darena + d.off_d;
  int32_t* I = iarena + d.off_i;
  int32_t* info = infos + size_t(blockIdx.x) * FPE_INFO_COUNT;
  const bool ref = d.disc == 0;

  if (threadIdx.x < FPE_INFO_COUNT) info[threadIdx.x] = 0;
  // ---- knots (thread 0) -------------------------------------------------
  if (threadIdx.x == 0) {
    int ns, nv;
    if (ref) {
      double center_s = (d.S0 - d.smin) / (d.smax - d.smin);
      ns = gen_knots_reference(S.knots[0], min(d.cap_knot_s, 512), d.n_s, center_s, d.smin, d.smax,
                               d.S0, 0.1, S.scratch);
      nv = gen_knots_reference(S.knots[1], min(d.cap_knot_v, 512), d.n_v, d.V0, d.vmin, d.vmax,
                               d.V0, 0.001, S.scratch);
    } else {
      ns = gen_knots_config(S.knots[0], min(d.cap_knot_s, 512), d.n_s, d.smin, d.smax, d.S0,
                            d.S0 / 5.0, true);
      nv = gen_knots_config(S.knots[1], min(d.cap_knot_v, 512), d.n_v, d.vmin, d.vmax, d.V0, 0.02,
                            false);
    }
    S.cnt[0] = ns;
    S.cnt[1] = nv;
  }
  __syncthreads();
  int nks = S.cnt[0], nkv = S.cnt[1];
  if (nks < 8 || nkv < 8) {
    if (threadIdx.x == 0) info[FPE_INFO_STATUS] = FPE_ERR_CAPACITY;
    return;
  }
  for (int i = threadIdx.x; i < nks; i += blockDim.x) D[DL.knot_s + i] = S.knots[0][i];
  for (int i = threadIdx.x; i < nkv; i += blockDim.x) D[DL.knot_v + i] = S.knots[1][i];

  // ---- quadrature grids and nodes per axis --------------------------------
  double glx[4], glw[4];
  gl4(ref, glx, glw);
  for (int ax = 0; ax < 2; ++ax) {
    const bool is_v = ax == 1;
    double* grid = D + (is_v ? DL.grid_v : DL.grid_s);
    const int cap_grid = is_v ? d.cap_grid_v : d.cap_grid_s;
    const int cap_q = is_v ? d.cap_q_v : d.cap_q_s;
    int ng = 0;
    if (ref) {
      if (threadIdx.x == 0) {
        int n = is_v ? grid_reference_raw(S.sortbuf, d.V0, 0.001, d.vmin, d.vmax, d.num_insert, true)
                     : grid_reference_raw(S.sortbuf, d.S0, 0.1, d.smin, d.smax, d.num_insert, false);
        S.cnt[2] = n;
      }
      __syncthreads();
      int n = S.cnt[2];
      int p2 = 1;
      while (p2 < n) p2 <<= 1;
      if (p2 > 8192) {
        if (threadIdx.x == 0) info[FPE_INFO_STATUS] = FPE_ERR_CAPACITY;
        return;
      }
      block_sort(S.sortbuf, n, p2);
      if (threadIdx.x == 0) {  // dedup exact duplicates (domain.mojo:68-75)
        int m = 0;
        for (int i = 0; i < n; ++i)
          if (m == 0 || S.sortbuf[i] != S.sortbuf[m - 1]) S.sortbuf[m++] = S.sortbuf[i];
        S.cnt[3] = m;
      }
      __syncthreads();
      ng = S.cnt[3];
      if (ng > cap_grid) {
        if (threadIdx.x == 0) info[FPE_INFO_STATUS] = FPE_ERR_CAPACITY;
        return;
      }
      if (!is_v) {  // normalize(s_grid_phys) (helpers.mojo:56-87)
        double mn = S.sortbuf[0], mx = S.sortbuf[ng - 1], range = mx - mn;
        double inv = range != 0.0 ? 1.0 / range : 0.0;
        for (int i = threadIdx.x; i < ng; i += blockDim.x)
          grid[i] = range != 0.0 ? (S.sortbuf[i] - mn) * inv : 0.0;
      } else {
        for (int i = threadIdx.x; i < ng; i += blockDim.x) grid[i] = S.sortbuf[i];
      }
    } else {
      // config: the distinct knots are the quadrature grid
      ng = is_v ? d.n_v : d.n_s;
      const double* kn = S.knots[ax];
      for (int i = threadIdx.x; i < ng; i += blockDim.x) grid[i] = kn[3 + i];
    }
    __syncthreads();
    const int per = ref ? 5 : 4;
    const int nq = (ng - 1) * per;
    if (nq > cap_q) {
      if (threadIdx.x == 0) info[FPE_INFO_STATUS] = FPE_ERR_CAPACITY;
      return;
    }
    double* qx = D + (is_v ? DL.qx_v : DL.qx_s);
    double* qw = D + (is_v ? DL.qw_v : DL.qw_s);
    double* qp = D + (is_v ? DL.qp_v : DL.qp_s);
    const double jac = is_v ? 1.0 : (d.smax - d.smin);
    for (int iv = threadIdx.x; iv < ng - 1; iv += blockDim.x) {
      double a = grid[iv], b = grid[iv + 1];
      double mid = (a + b) * 0.5, half = (b - a) * 0.5;
      int base = iv * per, k = 0;
      if (ref) {
        qx[base] = a;
        qw[base] = 0.0 * jac;
        k = 1;
      }
      for (int g = 0; g < 4; ++g) {
        qx[base + k + g] = mid + half * glx[g];
        qw[base + k + g] = (half * glw[g]) * jac;
      }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nq; q += blockDim.x)
      qp[q] = is_v ? qx[q] : d.smin + qx[q] * (d.smax - d.smin);
    if (threadIdx.x == 0) {
      info[is_v ? FPE_INFO_NGRID_V : FPE_INFO_NGRID_S] = ng;
      info[is_v ? FPE_INFO_NQ_V : FPE_INFO_NQ_S] = nq;
      info[is_v ? FPE_INFO_NKNOT_V : FPE_INFO_NKNOT_S] = is_v ? nkv : nks;
    }
    __syncthreads();

    // ---- recombined basis tables at the nodes --------------------------
    const double* kn = S.knots[ax];
    const int nk = is_v ? nkv : nks;
    const int ndof = nk - 4 - 2;
    const int cap_dof = is_v ? d.cap_dof_v : d.cap_dof_s;
    if (ndof > cap_dof || ndof < 4) {
      if (threadIdx.x == 0) info[FPE_INFO_STATUS] = FPE_ERR_CAPACITY;
      return;
    }
    const bool lneu = is_v ? true : d.left_neu != 0;
    const bool rneu = is_v ? true : d.right_neu != 0;
    double* Bt = D + (is_v ? DL.B_v : DL.B_s);
    double* dBt = D + (is_v ? DL.dB_v : DL.dB_s);
    int32_t* c0t = I + (is_v ? IL.c0_v : IL.c0_s);
    int32_t* rng = I + (is_v ? IL.rng_v : IL.rng_s);
    for (int c = threadIdx.x; c < ndof; c += blockDim.x) {
      rng[2 * c] = 0x7fffffff;
      rng[2 * c + 1] = -1;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nq; q += blockDim.x) {
      int c0;
      double B[4], dB[4];
      recombined_window(kn, nk, qx[q], lneu, rneu, &c0, B, dB);
      c0t[q] = c0;
      for (int k = 0; k < 4; ++k) {
        Bt[4 * q + k] = B[k];
        dBt[4 * q + k] = dB[k];
        if ((B[k] != 0.0 || dB[k] != 0.0) && c0 + k < ndof) {
          atomicMin(&rng[2 * (c0 + k)], q);
          atomicMax(&rng[2 * (c0 + k) + 1], q + 1);
        }
      }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < ndof; c += blockDim.x) {
      if (rng[2 * c + 1] < 0) {
        rng[2 * c] = 0;
        rng[2 * c + 1] = 0;
      }
    }
    if (threadIdx.x == 0) info[is_v ? FPE_INFO_NDOF_V : FPE_INFO_NDOF_S] = ndof;
    __syncthreads();
  }
  if (threadIdx.x == 0 &&
      (info[FPE_INFO_NDOF_V] > FPE_MAX_NDOF_V || info[FPE_INFO_NDOF_S] > FPE_MAX_NDOF_S))
    info[FPE_INFO_STATUS] = FPE_ERR_UNSUPPORTED;
}

}  // namespace fpe
