/*
 * ce_probe.h -- measurement helper exported by libce_gpu.so.
 *
 * No counterpart in the reference (its benchmarks are CPU-only). The explosion
 * kernel is bound by the FP32 CUDA-core pipe, not by tensor cores or HBM, so its
 * roofline denominator is the chip's FP32 FMA throughput, measured here with a
 * dependent-chain-free FFMA kernel (8 independent chains per thread, every SM
 * fully occupied), timed with CUDA events, best of 5.
 */
#ifndef CE_PROBE_H
#define CE_PROBE_H

#ifdef __cplusplus
extern "C" {
#endif

/* FP32 FMA throughput of `device` in TFLOP/s (an FMA counts 2), from a short
 * (~0.2 ms) scalar-FFMA kernel. Returns 0 or a negative CE_ERR_* code. */
int ce_probe_fp32_peak(int device, double* tflops_out);

/* The same throughput from a kernel sized to last at least `min_ms` (0 .. 1000)
 * milliseconds per launch, so the SM clock settles under load: scalar FFMA
 * (packed 0) or packed FFMA2 (packed 1, two FP32 FMAs per instruction with
 * per-element IEEE rounding, the form the explosion kernel's x/y components
 * use). Best of 5 timed launches after sizing. *ms_out (may be NULL) receives
 * the best launch's duration. Returns 0 or a negative CE_ERR_* code. */
int ce_probe_fp32_peak_ex(int device, int packed, double min_ms, double* tflops_out, double* ms_out);

/* Failure-detection check of the bounded waits the tensor-core kernels use
 * (no counterpart in the reference): one kernel waits on an mbarrier that
 * nothing arrives on, with at most `spins` polls (1 .. 2^20); the wait must give
 * up and record its error code (7) in *code_out while the context stays usable.
 * Returns 0 or a negative CE_ERR_* code. */
int ce_probe_bounded_wait(int device, unsigned spins, int* code_out);

#ifdef __cplusplus
}
#endif
#endif /* CE_PROBE_H */
