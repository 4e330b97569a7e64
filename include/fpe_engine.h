/** @file fpe_engine.h
 *  @brief C ABI of the B200 Heston Fokker-Planck pricing engine.
 *
 *  Part 1 is a drop-in for the reference C ABI (elevenwang-creator/FPE_option,
 *  cpp/include/fpe_engine.h): the same 16 symbols, argument order, struct
 *  layouts (sizes pinned by static_assert), ownership and error behaviour.
 *  Every result array is allocated by the library and released with the
 *  matching fpe_compute_free_* call; failures return NULL data and zero length.
 *
 *  Part 2 adds the batched entry points: thousands of contracts with
 *  different parameters, barriers and grid sizes priced in one launch
 *  sequence on one GPU.  There is no CPU fallback: when no CUDA device is
 *  usable every entry point fails (NULL handle / negative return code).
 */
#ifndef FPE_ENGINE_H
#define FPE_ENGINE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ======================= Part 1: reference C ABI ======================== */

/** Opaque handle to a stepwise pricing pipeline. */
typedef struct FpeCompute FpeCompute;

/** reference cpp/include/fpe_engine.h:21-24 */
struct FpeVecResult {
    double* data;
    int32_t len;
};

/** reference cpp/include/fpe_engine.h:27-32 */
struct FpeVec2Result {
    double* s_data;
    int32_t s_len;
    double* v_data;
    int32_t v_len;
};

/** reference cpp/include/fpe_engine.h:35-42 */
struct FpeGridPtsResult {
    double* s_data;
    int32_t s_len;
    double* v_data;
    int32_t v_len;
    double* sw_data;
    double* vw_data;
};

/** reference cpp/include/fpe_engine.h:45-49 (row-major) */
struct FpeMatResult {
    double* data;
    int32_t n_rows;
    int32_t n_cols;
};

/** reference cpp/include/fpe_engine.h:52-57 */
struct FpeGreeksResult {
    double* delta;
    double* gamma;
    double* vega;
    int32_t len;
};

/** reference cpp/include/fpe_engine.h:60-66 */
struct FpeOneshotResult {
    double* price;
    double* delta;
    double* gamma;
    double* vega;
    int32_t len;
};

/** Replaces reference fpe_compute_create (cpp/include/fpe_engine.h:87-94).
 *  s_min < 0 -> 0; s_max <= 0 -> 3*S0; num_insert <= 0 -> 251.
 *  Returns NULL on invalid parameters or when no GPU is usable. */
extern FpeCompute* fpe_compute_create(
    double kappa, double theta, double sigma, double rho,
    double r, double T, double S0, double V0,
    int32_t n_s, int32_t n_v,
    double barrier, int32_t option_type,
    int32_t num_insert,
    double s_min, double s_max);

/** Replaces reference fpe_compute_destroy (cpp/include/fpe_engine.h:97). */
extern void fpe_compute_destroy(FpeCompute* ptr);

/** Replaces reference fpe_compute_knots (cpp/include/fpe_engine.h:103). */
extern void fpe_compute_knots(FpeCompute* ptr, struct FpeVec2Result* result);

/** Replaces reference fpe_compute_grid_points (cpp/include/fpe_engine.h:109). */
extern void fpe_compute_grid_points(FpeCompute* ptr, struct FpeGridPtsResult* result);

/** Replaces reference fpe_compute_initial_condition (cpp/include/fpe_engine.h:115). */
extern void fpe_compute_initial_condition(FpeCompute* ptr, struct FpeVecResult* result);

/** Replaces reference fpe_compute_solve (cpp/include/fpe_engine.h:121):
 *  every accepted step (t = 0 included) x degrees of freedom, row-major. */
extern void fpe_compute_solve(FpeCompute* ptr, struct FpeMatResult* result);

/** Replaces reference fpe_compute_pdf (cpp/include/fpe_engine.h:127). */
extern void fpe_compute_pdf(FpeCompute* ptr, struct FpeMatResult* result);

/** Replaces reference fpe_compute_price (cpp/include/fpe_engine.h:135-140). */
extern void fpe_compute_price(FpeCompute* ptr, const double* K, int32_t n_K,
                              struct FpeVecResult* result);

/** Replaces reference fpe_compute_greeks (cpp/include/fpe_engine.h:150-157).
 *  rel_s / rel_v == 0 -> 0.01 / 0.1. */
extern void fpe_compute_greeks(FpeCompute* ptr, const double* K, int32_t n_K,
                               double rel_s, double rel_v, struct FpeGreeksResult* result);

/** Replaces reference fpe_price_oneshot (cpp/include/fpe_engine.h:164-173):
 *  price + central finite-difference Greeks (5 solves, 10 for knock-ins),
 *  all run as one batch. */
extern void fpe_price_oneshot(
    double kappa, double theta, double sigma, double rho,
    double r, double T, double S0, double V0,
    const double* K, int32_t n_K,
    double barrier, int32_t option_type,
    int32_t n_s, int32_t n_v,
    int32_t num_insert,
    double s_min, double s_max,
    struct FpeOneshotResult* result);

/** Replace reference fpe_compute_free_* (cpp/include/fpe_engine.h:176-186). */
extern void fpe_compute_free_vec(struct FpeVecResult* r);
extern void fpe_compute_free_vec2(struct FpeVec2Result* r);
extern void fpe_compute_free_grid_pts(struct FpeGridPtsResult* r);
extern void fpe_compute_free_mat(struct FpeMatResult* r);
extern void fpe_compute_free_greeks(struct FpeGreeksResult* r);
extern void fpe_compute_free_oneshot(struct FpeOneshotResult* r);

/* ================== Part 2: batched pricing (additions) ================= */

/** One contract.  option_type 0-9 as in the reference (down/up, in/out,
 *  call/put, european).  Knock-ins are priced by in-out parity (two solves).
 *  s_min < 0 -> 0; s_max <= 0 -> 3*S0. */
typedef struct FpeContract {
    double kappa, theta, sigma, rho, r, T, S0, V0;
    double barrier, s_min, s_max;
    int32_t n_s, n_v, option_type, n_strikes;
    const double* strikes;  /* host pointer, n_strikes values */
} FpeContract;

/** Batch options (zero-initialised = reference Pricer defaults in FP64). */
typedef struct FpeBatchOptions {
    int32_t disc;        /* 0 reference discretization, 1 config discretization */
    int32_t precision;   /* 0 FP64 stage factors, 1 FP32 factors + FP64 refinement */
    int32_t num_insert;  /* reference discretization grid size (<= 0 -> 50) */
    int32_t refine;      /* extra FP64 refinement sweeps per stage solve (<= 0 -> none:
                            the simplified Newton iteration's FP64 residual refines) */
    double rtol, atol;   /* Radau tolerances (<= 0 -> 1e-4 / 1e-6) */
    double ic_sigma_s, ic_sigma_v; /* config IC widths (<= 0 -> 0.6 / 0.004) */
    int32_t ic_sub;      /* config IC quadrature subintervals per span (<= 0 -> 8) */
    int32_t greeks;      /* 1: delta/gamma/vega by 4 bumped solves per contract */
    double rel_s, rel_v; /* Greeks bumps relative to S0 / V0 (<= 0 -> 0.01 / 0.1) */
    int32_t complex_solve; /* complex Radau stage: 0 auto (GMRES(10) for disc 0, direct
                              for disc 1), 1 GMRES(10) with the real-stage preconditioner
                              (the reference algorithm), 2 direct complex block LU */
    int32_t radau_constants; /* Radau IIA stage constants: 0 auto (the reference's
                                U1/ALPH/BETA/TI13 for disc 0, exact for disc 1),
                                1 the reference's, 2 exact (order-5 Radau IIA) */
    double max_step;     /* Radau step cap: <= 0 -> T/5 (the reference Pricer), > 0 absolute */
    double first_step;   /* first Radau step: 0 -> 1e-6 (the reference Pricer); < 0 -> the
                            solver's own estimate 0.01 / ||K y0 / scal|| (reference FPESolver
                            with first_step 0, src/numerics/ode/radau.mojo:168-184) */
    int32_t price_rule;  /* reference discretization only: 0 the Pricer's discounted
                            quadrature sum (pricer.mojo:27-64); 1 the calibration
                            objective's undiscounted sum over the quadrature points with
                            half-spacing weights, 1 at both ends
                            (src/engines/calibrator/objective.mojo:26-50) */
    int32_t max_steps;   /* accepted Radau steps before a solve ends with
                            FPE_STATUS_MAX_STEPS (<= 0 -> 100000, the reference cap,
                            src/numerics/ode/radau.mojo:257-263) */
    int32_t fp64_retry;  /* precision 1 only: a solve that ends with a solver failure
                            (FPE_STATUS_SINGULAR .. FPE_STATUS_TIMEOUT) is solved again
                            with FP64 factors and that attempt's price and status are
                            reported; 0 or 1 on (default), < 0 off */
    int64_t stage_wait_cycles; /* SM clock cycles a staged block solve waits for its
                            factor copies before the solve ends with FPE_STATUS_TIMEOUT
                            (<= 0 -> about one second); the FP64 retry always uses the
                            default.  A short limit exercises the failure path */
    int32_t block_split; /* stage-LU block size: 0 auto (the tuned choice per grid size,
                            else full nv x nv blocks when their factorization scratch fits
                            in shared memory, half-width blocks when not), 1 nv x nv
                            blocks, 2 (nv / 2) x (nv / 2) blocks (even nv) */
    int32_t sweep_buffers; /* stage buffers of the staged block solves: 0 auto (the tuned
                            choice, else 2), 2 .. 4 (as many as the shared scratch holds) */
    double knock_in_tol_scale; /* rtol and atol of both solves of a knock-in (in-out
                            parity) are multiplied by this: the price is the difference
                            of two larger prices, so their relative errors are amplified
                            by vanilla / knock-in.  <= 0 -> 1 on the reference
                            discretization (the reference Pricer), 0.01 on the config
                            discretization */
} FpeBatchOptions;

/** Status codes written per strike slot of a batch. */
#define FPE_STATUS_OK 0
#define FPE_STATUS_CAPACITY 1
#define FPE_STATUS_UNSUPPORTED 2
#define FPE_STATUS_SINGULAR 3
#define FPE_STATUS_MAX_STEPS 4
#define FPE_STATUS_STEP_UNDERFLOW 5
#define FPE_STATUS_NONFINITE 6
#define FPE_STATUS_TIMEOUT 7  /* a bounded device-side wait gave up (no reference counterpart) */
#define FPE_STATUS_INVALID 16

/** A prepared batch: descriptors and strikes resident on the device.
 *  No reference counterpart (the reference prices one contract per call). */
typedef struct FpePlan FpePlan;

/** Build a plan (host packing + one host-to-device copy). NULL on failure. */
extern FpePlan* fpe_plan_create(const FpeContract* contracts, int32_t n,
                                const FpeBatchOptions* opt);
/** Enqueue the whole solve pipeline on a CUDA stream (NULL = the library's
 *  stream); asynchronous.  Returns the number of kernel launches, < 0 on error. */
extern int32_t fpe_plan_run(FpePlan* plan, void* cuda_stream);
/** Wait for the plan, copy results to the host and combine parity / Greeks.
 *  Arrays hold one value per strike in contract order (delta/gamma/vega may
 *  be NULL; they are filled only when opt->greeks was set).  Returns 0 when
 *  every solve succeeded, otherwise the first non-zero status. */
extern int32_t fpe_plan_results(FpePlan* plan, double* prices, double* delta, double* gamma,
                                double* vega, int32_t* status);
/** Aggregated solver counters (20 slots): out[0] solves, [1] accepted steps,
 *  [2] rejected, [3] Newton iterations, [4] GMRES iterations, [5] LU
 *  factorizations, [6] ADMM iterations, [7] max n_dof_s, [8] max n_dof_v,
 *  [9] total dofs, [10] sweeps over real factors, [11] sweeps over complex
 *  factors, [12] algorithmic stage-factor bytes (written + read), [13] worst
 *  status, [14]-[17] SM kilo-cycles summed over solves spent in the Radau
 *  kernel's factorizations, block solves, Kronecker products and in total,
 *  [18]-[19] the parts of [14] spent in the pivot-block Gauss-Jordan
 *  eliminations and in the block products (L, W and Schur updates). */
extern int32_t fpe_plan_stats(FpePlan* plan, int64_t* out);
/** Run the pipeline once with a CUDA event around each of its five kernels
 *  (setup, galerkin, ic, radau, payoff); ms[5] receives the durations. */
extern int32_t fpe_plan_kernel_times(FpePlan* plan, void* cuda_stream, float* ms);
/** Number of strike results and of device solves in the plan. */
extern int32_t fpe_plan_sizes(FpePlan* plan, int32_t* n_results, int32_t* n_solves);
/** Solves of the last fpe_plan_results call that were solved again with FP64
 *  factors after a mixed-precision failure (opt->fp64_retry), or < 0. */
extern int32_t fpe_plan_retried(FpePlan* plan);
/** Tuned solve shape of a grid class, used by plans whose block_split /
 *  sweep_buffers options are 0 (auto).  No reference counterpart: the
 *  autotuner (fpe_option_b200/autotune.py) times the candidate shapes of each
 *  class on the device and installs the fastest here.  A class is (disc, n_s,
 *  n_v, precision, complex_solve) as in FpeContract / FpeBatchOptions;
 *  block_split 0 keeps the shared-memory fit rule.  The table can also be
 *  loaded at start-up from the text file named by the environment variable
 *  FPE_TUNE_TABLE (lines: disc n_s n_v precision complex_solve block_split
 *  sweep_buffers).  fpe_tune_set returns 0 or < 0 on a bad shape;
 *  fpe_tune_get returns 1 and fills the shape when the class is tuned, else 0. */
extern int32_t fpe_tune_set(int32_t disc, int32_t n_s, int32_t n_v, int32_t precision, int32_t complex_solve,
                            int32_t block_split, int32_t sweep_buffers);
extern int32_t fpe_tune_get(int32_t disc, int32_t n_s, int32_t n_v, int32_t precision, int32_t complex_solve,
                            int32_t* block_split, int32_t* sweep_buffers);
extern void fpe_tune_clear(void);

/** Number of words per solve in fpe_plan_solve_info. */
#define FPE_SOLVE_INFO_WORDS 40
/** Per-solve counters of the plan's last run, FPE_SOLVE_INFO_WORDS words per
 *  solve in the plan's solve order (longest estimated solve first): 0 status,
 *  7-8 dofs (s, v), 9 accepted, 10 rejected, 11 Newton, 12 GMRES, 13 LU
 *  factorizations, 14 ADMM iterations, 15 / 17 real / complex sweeps,
 *  18-21 SM kilo-cycles in factorizations, block solves, Kronecker products
 *  and in total, 22-23 the factorization's pivot inverses and block
 *  products, 24 the sweeps' waits for their factor copies, 25-27 the
 *  overlapped factorization phase's own work of the real pivot inverse, the
 *  complex pivot inverse and the other Schur updates, 28 the stage
 *  matrices' assembly, 29 the block rows' staging and pivot-inverse
 *  extraction, 30-32 the sweeps' stage work of a real row and of a complex
 *  row and a real row's wait at the stage barriers.  out holds
 *  n_solves * FPE_SOLVE_INFO_WORDS words.  Returns n_solves, < 0 on error. */
extern int32_t fpe_plan_solve_info(FpePlan* plan, int32_t* out);
extern void fpe_plan_destroy(FpePlan* plan);

/** One-call batch: plan, run, results, destroy. */
extern int32_t fpe_price_batch(const FpeContract* contracts, int32_t n,
                               const FpeBatchOptions* opt, double* prices, double* delta,
                               double* gamma, double* vega, int32_t* status);

/** Stepwise pipeline with explicit options (the reference create uses Compute
 *  defaults: reference discretization, rtol 1e-4, atol 1e-6). */
extern FpeCompute* fpe_compute_create_ex(
    double kappa, double theta, double sigma, double rho,
    double r, double T, double S0, double V0,
    int32_t n_s, int32_t n_v, double barrier, int32_t option_type,
    double s_min, double s_max, const FpeBatchOptions* opt);

/** Recombined 1-D basis of a pipeline as CSR (which: 0 Bs, 1 dBs, 2 Bv, 3 dBv);
 *  returns nnz; arrays are filled when non-NULL. */
extern int64_t fpe_compute_basis_csr(FpeCompute* ptr, int32_t which, int32_t* n_rows,
                                     int32_t* n_cols, int32_t* indptr, int32_t* indices,
                                     double* data);

/** Device availability: 1 when a CUDA device can run the kernels. */
extern int32_t fpe_device_available(void);

/** Returned by fpe_price_noalloc when a contract's grids need more scratch than
 *  its static array holds (or n_strikes is outside 1..1024). */
#define FPE_NOALLOC_ERR_SIZE (-2)
/** Returned by fpe_price_noalloc when cuda_stream is being captured into a
 *  CUDA graph; nothing was enqueued and the capture is left intact. */
#define FPE_NOALLOC_ERR_CAPTURE (-3)

/** Price one contract without allocating any memory.
 *
 *  No counterpart in the reference (which allocates per call).  For callers
 *  that cannot allocate device memory while pricing: hosts whose GPU memory
 *  budget is fixed at start-up, and plug-ins inside an application that owns
 *  the device memory pool.  All device scratch comes from one static device
 *  array of 64 MiB, held by every GPU that loads the library until exit; a
 *  contract whose grids need more (large n_s x n_v) is rejected with
 *  FPE_NOALLOC_ERR_SIZE and its status slots set to FPE_STATUS_CAPACITY.  The
 *  first call on each device (the current one) sets that device up: the
 *  array's device address, a stream of its own, the kernels' shared-memory
 *  limits.  Calls share the array: overlapping calls on one device race and
 *  must be serialized by the caller.  The call copies prices / status
 *  (n_strikes values, host memory) back and waits for its stream, so it cannot
 *  run on a stream under graph capture: such a stream gives
 *  FPE_NOALLOC_ERR_CAPTURE before anything is enqueued.  Knock-ins use in-out
 *  parity; opt->greeks must be 0; opt->fp64_retry is not applied.  Runs on
 *  cuda_stream (NULL: the device's own stream).  Returns 0, a status code, or
 *  < 0. */
extern int32_t fpe_price_noalloc(const FpeContract* contract, const FpeBatchOptions* opt,
                                 double* prices, int32_t* status, void* cuda_stream);

/** European prices from the Heston characteristic function (Heston 1993
 *  probabilities in the Albrecher et al. 2007 form, composite 16-point
 *  Gauss-Legendre quadrature), FP64, one warp per price.
 *
 *  No counterpart in the reference, which has no closed-form price; it
 *  measures the discretization error of the FPE prices of Europeans and prices
 *  European quotes directly.  Device pointers: params_dev holds n rows of 8
 *  values (kappa, theta, sigma, rho, r, T, S0, V0), strikes_dev n strikes,
 *  put_dev n flags (non-zero: put by put-call parity; NULL: all calls);
 *  prices_dev receives n prices, NaN for a row outside the model's domain.
 *  Asynchronous on cuda_stream (NULL: the library's stream).  Returns 0, or
 *  < 0 on a bad argument or CUDA error. */
extern int32_t fpe_heston_cf_batch(const double* params_dev, const double* strikes_dev,
                                   const int32_t* put_dev, int32_t n, double* prices_dev,
                                   void* cuda_stream);

/** The same prices for host contracts, one per strike in contract order like
 *  fpe_price_batch (grid fields are ignored).  Option types 8 (call) and 9
 *  (put) only: other types get FPE_STATUS_UNSUPPORTED, invalid parameters
 *  FPE_STATUS_INVALID, and NaN prices.  Synchronous; returns 0, the first
 *  non-zero status, or < 0 on a bad argument or CUDA error. */
extern int32_t fpe_heston_cf_price(const FpeContract* contracts, int32_t n, double* prices,
                                   int32_t* status);

/** Terminal density interpolated at n points (s, v), FP64, one thread per
 *  point: Catmull-Rom bicubic on the 4 x 4 neighbourhood of the enclosing
 *  cell (indices clamped at the edges, local coordinates clamped to [0, 1]),
 *  bilinear when either axis has fewer than 4 points.
 *
 *  Replaces reference Interpolator.interpolate / interpolate_batch
 *  (src/server/interpolator.mojo:62-198), which has no entry point of its
 *  own in the reference API.  Device pointers: the grid axes (nondecreasing,
 *  n_s and n_v >= 2), the density row-major n_s x n_v (as fpe_compute_pdf
 *  returns it, on the points of fpe_compute_grid_points), the query
 *  coordinates and out (n values).  Asynchronous on cuda_stream (NULL: the
 *  library's stream).  Returns 0, or < 0 on a bad argument or CUDA error. */
extern int32_t fpe_pdf_interpolate(const double* s_points_dev, int32_t n_s, const double* v_points_dev,
                                   int32_t n_v, const double* pdf_dev, const double* s_dev,
                                   const double* v_dev, int32_t n, double* out_dev, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
static_assert(sizeof(struct FpeVecResult) == 16, "FpeVecResult layout mismatch");
static_assert(sizeof(struct FpeVec2Result) == 32, "FpeVec2Result layout mismatch");
static_assert(sizeof(struct FpeGridPtsResult) == 48, "FpeGridPtsResult layout mismatch");
static_assert(sizeof(struct FpeMatResult) == 16, "FpeMatResult layout mismatch");
static_assert(sizeof(struct FpeGreeksResult) == 32, "FpeGreeksResult layout mismatch");
static_assert(sizeof(struct FpeOneshotResult) == 40, "FpeOneshotResult layout mismatch");
#endif

#endif
