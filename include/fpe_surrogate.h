/*
 * Surrogate pricer: a small MLP (n_in -> hidden x layers -> 1, SiLU) with BF16
 * weights and activations, FP32 accumulation, trained by Adam on prices made
 * by the batched FPE solver.  Its dense layers run on the B200's tensor cores
 * (tcgen05 MMA into tensor memory).  It has no counterpart in the reference
 * engine except the Adam update rule (reference src/nn/adam.mojo:31-64: bias
 * correction, epsilon added to the square root of the corrected second moment).
 *
 * All pointers named *_dev are device pointers; the caller owns them.  A
 * handle is not thread-safe; distinct handles are independent.  Every call
 * returns 0 on success and a negative value on a bad argument or CUDA error.
 */
#ifndef FPE_SURROGATE_H
#define FPE_SURROGATE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct FpeMlp FpeMlp;

/** Creates a network with n_in inputs (padded internally to a multiple of 16),
 *  `layers` hidden layers of width `hidden` (128 or 256: the weight-gradient
 *  products tile the hidden dimension by 128 tensor-memory lanes) and
 *  one output, training on up to `max_rows` rows per step; inference takes any
 *  number of rows, in launch sequences of max(max_rows, 65536) rows.  Weights are initialised like
 *  a default linear layer, U(-1/sqrt(fan_in), 1/sqrt(fan_in)), from `seed`.
 *  Returns NULL on a bad argument or without a GPU. */
extern FpeMlp* fpe_mlp_create(int32_t n_in, int32_t hidden, int32_t layers, int32_t max_rows,
                              uint64_t seed);
extern void fpe_mlp_destroy(FpeMlp* mlp);

/** layout[4] = {n_in, n_in padded, hidden, layers}; returns the number of
 *  parameters.  Parameters are FP32, flattened per hidden layer as the weight
 *  (hidden x n_in padded, row-major; padded columns stay zero) then the bias,
 *  followed by the output weights (hidden) and the output bias. */
extern int64_t fpe_mlp_layout(const FpeMlp* mlp, int32_t* layout);
extern int32_t fpe_mlp_get_params(FpeMlp* mlp, float* host_out, int64_t n);
/** Sets the FP32 master parameters and resets the Adam state. */
extern int32_t fpe_mlp_set_params(FpeMlp* mlp, const float* host_in, int64_t n);

/** y_dev[n] = network(x_dev[n x n_in]) on `cuda_stream` (NULL: the library's). */
extern int32_t fpe_mlp_forward(FpeMlp* mlp, const float* x_dev, int32_t n, float* y_dev,
                               void* cuda_stream);

/** One Adam step (learning rate lr, beta1 0.9, beta2 0.999, eps 1e-8) on the
 *  weighted squared error  sum_i w_i (y_hat_i - y_i)^2 / n  over n <= max_rows
 *  rows; w_dev may be NULL (weights 1).  loss_dev (optional, device float)
 *  receives the loss before the step.  lr < 0 takes the rate of the current
 *  step from the schedule set by fpe_mlp_set_lr_schedule.  The step counter
 *  and bias corrections live on the device and the call makes no host
 *  synchronisation, so a sequence of steps can be captured in a CUDA graph on
 *  a caller's stream and replayed. */
extern int32_t fpe_mlp_train_step(FpeMlp* mlp, const float* x_dev, const float* y_dev,
                                  const float* w_dev, int32_t n, float lr, float* loss_dev,
                                  void* cuda_stream);

/** Learning-rate schedule: entry t - 1 is the rate of Adam step t (the last
 *  entry repeats); n = 0 clears it.  Copied to the device. */
extern int32_t fpe_mlp_set_lr_schedule(FpeMlp* mlp, const float* host_table, int32_t n);

/** Gradient of the same loss at the current parameters, copied to
 *  grad_host[n_params] (no update); *loss_host receives the loss. */
extern int32_t fpe_mlp_gradient(FpeMlp* mlp, const float* x_dev, const float* y_dev,
                                const float* w_dev, int32_t n, float* grad_host, float* loss_host);

/** Tensor-core product C[M x N] = A[M x K] B[N x K]^T of BF16 row-major
 *  operands (lda, ldb in elements, multiples of 8; M a multiple of 128, N and
 *  K multiples of 16), FP32 accumulation, FP32 row-major result (ldc), plus
 *  bias[N] when bias_dev is not NULL; act = 1 applies SiLU. */
extern int32_t fpe_gemm_bf16(const void* a_dev, int32_t lda, const void* b_dev, int32_t ldb,
                             int32_t M, int32_t N, int32_t K, const float* bias_dev, int32_t act,
                             float* c_dev, int32_t ldc, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* FPE_SURROGATE_H */
