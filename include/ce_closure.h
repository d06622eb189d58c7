/*
 * ce_closure.h -- learned asymptotic closure of libce_gpu.so: a BF16 MLP with
 * FP32 accumulation, trained and served by hand-written sm_100a tensor-core
 * kernels (tcgen05.mma, accumulators in tensor memory).
 *
 * No counterpart in the reference: its only "closure" is the uniform velocity
 * rescale that moves the residual potential energy into kinetic energy at the
 * stop (src/driver.cpp:38-42). The engine stops integration early (at a loose
 * potential-energy fraction), adds the analytic straight-line (ballistic)
 * impulse of every pair from the stop to t -> infinity, and the network predicts
 * the remaining correction; a per-sim energy and momentum check sends doubtful
 * sims back to plain integration.
 */
#ifndef CE_CLOSURE_H
#define CE_CLOSURE_H

#include <stddef.h>
#include <stdint.h>

#include "ce_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- the network ----------------------------------------------------------
 * in_dim -> hidden (x depth, SiLU) -> out_dim, weights [fan_out][fan_in]
 * (row-major, BF16 copy of FP32 master weights), biases FP32. in_dim, hidden
 * and out_dim multiples of 16, hidden and out_dim <= 256. Batches are
 * multiples of 128 rows up to max_batch. Parameters are laid out
 * [W_0, b_0, W_1, b_1, ...] in ce_mlp_get_params / ce_mlp_set_params. */
typedef struct ce_mlp ce_mlp;
int ce_mlp_create(ce_mlp** out, int device, int in_dim, int hidden, int depth, int out_dim, uint64_t max_batch,
                  uint64_t seed);
void ce_mlp_destroy(ce_mlp* n);
const char* ce_mlp_last_error(const ce_mlp* n);
uint64_t ce_mlp_param_count(const ce_mlp* n);
int ce_mlp_set_params(ce_mlp* n, const float* host);
int ce_mlp_get_params(const ce_mlp* n, float* host);
/* x: [B][in_dim] BF16 (device), out: [B][out_dim] FP32 (device). Async on stream. */
int ce_mlp_forward(ce_mlp* n, const void* x, uint64_t B, float* out, void* stream);
/* Loss = sum(weight * (out - target)^2) with weights summing to 1 over the batch
 * (target, weight: [B][out_dim] FP32, device). Synchronous: writes the loss and,
 * if grads_host is not NULL, the FP32 gradients in parameter layout. */
int ce_mlp_gradients(ce_mlp* n, const void* x, const float* target, const float* weight, uint64_t B, float* loss,
                     float* grads_host, void* stream);
/* One Adam step (lr; beta 0.9 / 0.999, eps 1e-8). Async; if loss_dev is not
 * NULL the step's loss is copied there (device float). */
int ce_mlp_train_step(ce_mlp* n, const void* x, const float* target, const float* weight, uint64_t B, float lr,
                      float* loss_dev, void* stream);
/* Synchronise and report whether any tensor-core wait timed out. */
int ce_mlp_check(ce_mlp* n, void* stream);

/* Tensor-core GEMM used by the network, exposed for tests: C[M][N] (FP32) =
 * A B^T with BF16 A given K-major ([M][K]) or MN-major ([K][M]), B likewise
 * ([N][K] or [K][N]); N multiple of 16, M and K multiples of 8. *err_dev is set
 * non-zero if a tensor-core wait timed out. */
int ce_umma_gemm_f32(const void* A, int a_mn, const void* B, int b_mn, int M, int N, int K, float* C, int* err_dev,
                     void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CE_CLOSURE_H */
