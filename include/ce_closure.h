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
/* Serving forward. x: [B][in_dim] BF16 (device), out: [B][out_dim] FP32
 * (device); async on stream. When every layer is at most 256 wide and a
 * multiple of 32, with at most 8 layers, one fused persistent kernel runs the
 * whole network and B may be any multiple of 128 up to 2^30 (else B <=
 * max_batch and the per-layer path below is used). Both paths round at the
 * same points, so they agree bit for bit. */
int ce_mlp_forward(ce_mlp* n, const void* x, uint64_t B, float* out, void* stream);
/* The per-layer forward of the training path (B <= max_batch), for tests. */
int ce_mlp_forward_layered(ce_mlp* n, const void* x, uint64_t B, float* out, void* stream);
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

/* Shape of a network (any pointer may be NULL). */
int ce_mlp_shape(const ce_mlp* n, int* in_dim, int* hidden, int* depth, int* out_dim, uint64_t* max_batch);

/* Tensor-core GEMM used by the network, exposed for tests: C[M][N] (FP32) =
 * A B^T with BF16 A given K-major ([M][K]) or MN-major ([K][M]), B likewise
 * ([N][K] or [K][N]); N multiple of 16, M and K multiples of 8. *err_dev is set
 * non-zero if a tensor-core wait timed out. */
int ce_umma_gemm_f32(const void* A, int a_mn, const void* B, int b_mn, int M, int N, int K, float* C, int* err_dev,
                     void* stream);

/* ---- the closure around the mixed-batch engine ---------------------------
 * Rows are the mixed layout of ce_gpu.h (10 atoms per sim). Per sim the
 * network sees CE_CLOSURE_FEATURES BF16 inputs: per atom i < 10 the 12 values
 * (x_i - x_com)/L (3), p_i/P (3), (p_base,i - p_i)/P (3), q_i/3,
 * ln(m_i / amu)/3.5, 1 (zeros for the padded atoms), then PE_stop/E_0 * 20,
 * n/10 and zeros; L is the RMS distance from the centre of mass, P the RMS
 * atom momentum of the base p_base. It predicts CE_CLOSURE_OUTPUTS values, the
 * first 3n being (p_inf - p_base)/Q, Q = RMS over atoms of |p_base,i - p_i|
 * (the size of the analytic step). */
#define CE_CLOSURE_FEATURES 128
#define CE_CLOSURE_OUTPUTS 32

/* State at the loose stop, as ce_run_mixed_device writes it with
 * redistribute_energy = 0 (device pointers, mixed layout). */
typedef struct ce_closure_state {
  const float* positions;  /* [S][10][3] */
  const float* momenta;    /* [S][10][3] m v, no energy rescale */
  const double* e0;        /* [S] E_0 = PE_0 */
  const double* pe_final;  /* [S] PE at the stop */
  const uint8_t* status;   /* [S] CE_SIM_* of the loose run */
} ce_closure_state;

/* Bounds a sim's corrected momenta p = p_base + Q * out must meet to be
 * accepted (else it is integrated again by plain RK45):
 *   |KE(p)/E_0 - 1|            <= tol_energy      (energy conservation)
 *   |sum_i p_i| / sum_i |p_i|   <= tol_momentum    (momentum conservation)
 *   |Q * out| / |p_base|        <= tol_correction  (size of the learned step) */
typedef struct ce_closure_gate {
  float tol_energy;
  float tol_momentum;
  float tol_correction;
} ce_closure_gate;
void ce_closure_default_gate(ce_closure_gate* g);

/* Features, ballistic base and (if target != NULL) training targets for S sims
 * (device pointers, async on stream). feats [pad128(S)][128] BF16 (padded rows
 * zeroed); p_base [S][10][3]; p_scale [S] = Q (0 for one-atom or unconverged
 * sims, NaN when the ballistic integral does not exist); target, weight
 * [pad128(S)][32] FP32 with target = (p_true - p_base)/Q and, on the 3n live
 * components (zero elsewhere), weight = weight_scale / (3n) * 1e-2 /
 * sqrt(rms^2 + (1e-4)^2) where rms is the sim's RMS target: a relative loss. */
int ce_closure_features(uint64_t S, const ce_mixed_batch* in, double coulomb_k, const ce_closure_state* st,
                        const float* p_true, float weight_scale, void* feats, float* p_base, float* p_scale,
                        float* target, float* weight, void* stream);

/* Gate and final momenta from the network output [pad128(S)][32]: accepted
 * sims get p projected to zero net momentum (mass weighted) and rescaled to
 * KE = E_0, status CE_SIM_OK and the loose run's step count; sims with n < 2
 * copy the loose run's status and zero momenta; every other sim gets
 * fallback[s] = n (else 0) and its outputs are left untouched. counts[0] +=
 * accepted, counts[1] += sent back. */
int ce_closure_apply(uint64_t S, const ce_mixed_batch* in, const ce_closure_state* st, const uint32_t* steps_loose,
                     const float* p_base, const float* p_scale, const float* net_out, const ce_closure_gate* gate,
                     const ce_outputs* out, uint8_t* fallback, unsigned long long* counts, void* stream);

/* Serving pipeline bound to one engine and one network (in_dim 128, out_dim 32):
 * loose run (cfg with pe_stop_fraction = loose_pe_stop and no rescale, keeping
 * each sim's integrator state, ce_sim_state) -> features -> network -> gate ->
 * plain RK45 (cfg) for the sims sent back, continued from their loose-stop
 * state, so their results are bit for bit those of plain RK45 (a sim whose loose
 * run failed restarts from rest) -> merge. Device pointers, stream-ordered, no host synchronisation and no
 * allocation (scratch for max_sims sims is allocated by ce_closure_create), so
 * a call can be captured in a CUDA graph. out->momenta/ker/steps/status are
 * written (other fields ignored). */
typedef struct ce_closure ce_closure;
int ce_closure_create(ce_closure** out, ce_engine* e, ce_mlp* net, uint64_t max_sims);
void ce_closure_destroy(ce_closure* c);
const char* ce_closure_last_error(const ce_closure* c);
int ce_closure_serve(ce_closure* c, uint64_t S, const ce_mixed_batch* in, double coulomb_k, const ce_run_config* cfg,
                     double loose_pe_stop, const ce_closure_gate* gate, const ce_outputs* out, void* stream);
/* Synchronise the last serve's stream and read its accepted / sent-back counts. */
int ce_closure_counts(ce_closure* c, uint64_t* accepted, uint64_t* fallback);
/* Copy (device to device, async on stream) the last serve's per-sim flags:
 * n for each sim sent back to plain integration, 0 otherwise. S <= max_sims. */
int ce_closure_fallback_flags(const ce_closure* c, uint8_t* dst, uint64_t S, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CE_CLOSURE_H */
