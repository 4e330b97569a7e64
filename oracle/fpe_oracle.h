/* CPU FP64 oracle for the Heston Fokker-Planck pricing path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain-C++ restatement of the
 * reference Mojo CPU engine (elevenwang-creator/FPE_option, src/engines/fpe,
 * src/numerics, src/server).  It is used by tests/ as the parity checker and by
 * bench.py as the timed CPU baseline.  The product (fpe_option_b200) never
 * links, loads or calls it.
 *
 * Two discretizations share one engine:
 *   disc = 0  "reference": knot, quadrature, IC and BC rules of the Mojo engine
 *   disc = 1  "config"   : sinh-stretched clamped knots, 4-point Gauss-Legendre
 *                          per knot span, wide bivariate-normal IC, exact payoff
 *                          integration (the workload definition of the batched
 *                          benchmarks).
 */
#ifndef FPE_ORACLE_H
#define FPE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrcPipeline OrcPipeline;

/* Solver / discretization options (zero-initialised struct = reference defaults
 * of ComputePipeline: num_insert 251, rtol 1e-4, atol 1e-6, disc 0). */
typedef struct OrcOptions {
    int32_t disc;          /* 0 reference, 1 config */
    int32_t num_insert;    /* reference disc: quadrature grid size (<=0 -> 251) */
    double rtol;           /* <=0 -> 1e-4 */
    double atol;           /* <=0 -> 1e-6 */
    double ic_sigma_s;     /* config disc IC width in s (<=0 -> 0.6) */
    double ic_sigma_v;     /* config disc IC width in v (<=0 -> 0.004) */
    int32_t nnls_exact;    /* 1: solve the IC NNLS to optimality instead of ADMM */
    int32_t ic_sub;        /* config disc: IC quadrature subintervals per span (<=0 -> 8) */
    int32_t complex_direct; /* 1: exact complex stage solve instead of GMRES(10) */
    int32_t radau_constants; /* 0 auto (reference for disc 0, exact for disc 1),
                                1 the reference's U1/ALPH/BETA, 2 exact Radau IIA */
    double max_step;       /* <=0 -> T/5 (Pricer, pricer.mojo:131-136); >0 absolute */
    double first_step;     /* 0 -> 1e-6 (Pricer); <0 -> the solver's own estimate
                              (radau.mojo:168-184, FPESolver first_step=0); >0 as given */
    int32_t price_rule;    /* reference disc: 0 Pricer._price_at (discounted quadrature
                              sum); 1 the calibration objective's undiscounted sum with
                              half-spacing weights (objective.mojo:26-50) */
} OrcOptions;

/* ComputePipeline(fp, num_insert) (reference src/server/compute_pipeline.mojo:29-48).
 * Returns NULL when the parameters are invalid (FpeParams.is_valid). */
OrcPipeline* orc_create(double kappa, double theta, double sigma, double rho,
                        double r, double T, double S0, double V0,
                        int32_t n_s, int32_t n_v, double barrier, int32_t option_type,
                        double s_min, double s_max, const OrcOptions* opt);
void orc_destroy(OrcPipeline* p);

/* Array access.  what: 0 s-knots, 1 v-knots, 2 s points (phys), 3 v points,
 * 4 s weights, 5 v weights, 6 initial condition q0, 7 terminal coefficients q_T,
 * 8 full trajectory (n_saved x N, row-major), 9 pdf (n_qs x n_qv),
 * 10 saved times, 11 D scaling vector, 12 galerkin projection b.
 * orc_len returns the element count; orc_fill copies into out (caller-sized). */
int64_t orc_len(OrcPipeline* p, int32_t what);
int64_t orc_fill(OrcPipeline* p, int32_t what, double* out);

/* Dimensions: out[0]=n_dof_s out[1]=n_dof_v out[2]=n_qs out[3]=n_qv
 * out[4]=accepted steps out[5]=rejected steps out[6]=newton iterations
 * out[7]=gmres iterations out[8]=lu factorizations out[9]=admm iterations
 * out[10]=solve success (1/0) out[11]=band half-width kl. Triggers the solve. */
void orc_dims(OrcPipeline* p, int64_t* out);

/* 1-D basis CSR export (which: 0 Bs, 1 dBs, 2 Bv, 3 dBv). Returns nnz, fills
 * arrays when non-NULL (indptr has nrows+1 entries). */
int64_t orc_basis_csr(OrcPipeline* p, int32_t which, int32_t* nrows, int32_t* ncols,
                      int32_t* indptr, int32_t* indices, double* data);

/* 1-D Galerkin factor export, dense row-major n x n (which: 0 Ns, 1 Ss=dBs^T diag(s w) Bs,
 * 2 Tss=dBs^T diag(s^2 w) dBs, 3 Nv, 4 V2, 5 V3, 6 V4, 7 V5, 8 V6). Returns n. */
int32_t orc_factor(OrcPipeline* p, int32_t which, double* out);

/* ComputePipeline.price_at / greeks (compute_pipeline.mojo:116-171). */
int32_t orc_price_at(OrcPipeline* p, const double* K, int32_t nK, double* out);
int32_t orc_greeks(OrcPipeline* p, const double* K, int32_t nK, double rel_s, double rel_v,
                   double* delta, double* gamma, double* vega);

/* Pricer(rtol, atol, num_insert).price(fp) (pricer.mojo:82-155), in-out parity
 * included.  Returns 0 on success, -1 on invalid parameters (prices zeroed). */
int32_t orc_pricer_price(double kappa, double theta, double sigma, double rho,
                         double r, double T, double S0, double V0,
                         int32_t n_s, int32_t n_v, double barrier, int32_t option_type,
                         double s_min, double s_max, const double* K, int32_t nK,
                         const OrcOptions* opt, double* out);

/* PricingEngine(num_insert).price(fp) = price + Greeks (pricing_engine.mojo:16-52). */
int32_t orc_engine_price(double kappa, double theta, double sigma, double rho,
                         double r, double T, double S0, double V0,
                         int32_t n_s, int32_t n_v, double barrier, int32_t option_type,
                         double s_min, double s_max, const double* K, int32_t nK,
                         const OrcOptions* opt,
                         double* price, double* delta, double* gamma, double* vega);

/* Batch of independent contracts (one strike each), spread over n_threads host
 * threads, one contract per thread at a time.  params: n x 12 row-major
 * [kappa theta sigma rho r T S0 V0 K barrier s_min s_max]; ints: n x 3
 * [n_s n_v option_type]. */
int32_t orc_price_batch(int32_t n, const double* params, const int32_t* ints,
                        const OrcOptions* opt, int32_t n_threads, double* out);

/* FP64 Heston characteristic-function European price (Albrecher et al. 2007
 * "little Heston trap" form), Gauss-Legendre on a truncated integration range. */
/* Interpolator.interpolate over n points (src/server/interpolator.mojo:62-198):
 * Catmull-Rom bicubic, bilinear below 4 points per axis; pdf row-major n_s x n_v. */
int32_t orc_pdf_interpolate(const double* s_points, int32_t n_s, const double* v_points, int32_t n_v,
                            const double* pdf, const double* s, const double* v, int32_t n, double* out);

double orc_heston_cf_price(double kappa, double theta, double sigma, double rho,
                           double r, double T, double S0, double V0, double K,
                           int32_t is_call);

/* Component-level helpers used by unit tests against the reference's own tests. */
double orc_bspline_value(const double* knots, int32_t n_knots, int32_t degree,
                         double x, int32_t i);
int32_t orc_generate_knots(int32_t n, int32_t degree, int32_t nonuniform, double center,
                           double b0, double b1, double mean, double std_, double* out);
int32_t orc_payoff(int32_t option_type, const double* K, int32_t nK, double barrier,
                   double S, double* out);
/* Radau IIA on M y' = -K y with dense M, K (n x n row-major); returns accepted
 * steps (-1 on failure).  exact_constants selects the true Radau IIA eigenvalues
 * instead of the reference's hard-coded U1/ALPH/BETA. */
int32_t orc_radau_dense(int32_t n, const double* M, const double* K, const double* y0,
                        double t1, double rtol, double atol, double max_step,
                        double first_step, int32_t exact_constants, double* y_out);

#ifdef __cplusplus
}
#endif
#endif
