/*
 * ce_oracle.h -- CPU oracle for the batched Coulomb-explosion path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker, never the product: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it.
 * The product path (libce_gpu.so) neither links nor calls anything here.
 *
 * A plain-C restatement of the reference scalar engine, in both precisions:
 *   - pair force / potential / kinetic energy   src/system.cpp:5-49
 *   - adaptive Dormand-Prince DP5(4) step        src/integrators.cpp:63-147
 *   - Hairer initial step                        src/integrators.cpp:197-250
 *   - convergence driver + redistribution        src/driver.cpp:7-46
 * The operation order follows those lines so that, compiled without FMA
 * contraction, the f32/f64 results are bit-identical to the reference engine
 * built from its own sources (pinned by tests/test_oracle_pin.py).
 *
 * Two optional forms that have no reference counterpart restate the GPU
 * engine's precision modes (selected by ce_oracle_cfg.mode bits):
 *   CE_ORACLE_KAHAN : compensated (Kahan) accumulation of the accepted x/v updates
 *   CE_ORACLE_FP64  : FP64 time accumulator, FP64 potential-energy sum for the
 *                     convergence check, FP64 finalize (the batched engine's
 *                     finalize policy, include/coulomb/batched_integrator.hpp:172-189)
 */
#ifndef CE_ORACLE_H
#define CE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CE_ORACLE_KAHAN 1
#define CE_ORACLE_FP64 2

/* Per-sim outcome, same codes as the reference precision sweep's FailureCode
 * (bench/bench_precision_sweep.cpp:80-85). */
#define CE_ORACLE_OK 0
#define CE_ORACLE_REJECT_LIMIT 1 /* integrator threw: > 100 rejections */
#define CE_ORACLE_MAX_STEPS 2    /* hit max_steps before pe_stop */
#define CE_ORACLE_NONFINITE 3    /* NaN/Inf in the final momenta */

typedef struct ce_oracle_cfg {
  double rtol;             /* IntegratorOptions::rtol (integrator.hpp:231)        */
  double atol;             /* IntegratorOptions::atol (integrator.hpp:232)        */
  double pe_stop_fraction; /* RunConfig::pe_stop_fraction (driver.hpp:147)        */
  double max_dt;           /* RunConfig::max_dt (driver.hpp:159)                  */
  uint64_t max_steps;      /* RunConfig::max_steps (driver.hpp:162)               */
  int redistribute_energy; /* RunConfig::redistribute_energy (driver.hpp:155)     */
  int mode;                /* 0 = reference semantics; bits CE_ORACLE_KAHAN|FP64  */
  int integrator;          /* 0 = DP5(4); 1 = Velocity Verlet with the fixed step
                              max_dt (src/integrators.cpp:14-47; mode must be 0)   */
} ce_oracle_cfg;

typedef struct ce_oracle_stats {
  uint32_t steps;   /* accepted steps (RunResult::steps)                    */
  uint32_t rejects; /* rejected attempts over the whole run                 */
  uint8_t status;   /* CE_ORACLE_*                                           */
  double t_final, e0, pe_final, ke_before, ke_after, scale;
} ce_oracle_stats;

/* Accelerations a[n][3] of one configuration (system.cpp:5-29). */
void ce_oracle_accel_f64(int n, const double* x, const double* mass, const double* charge,
                         double coulomb_k, double* a);
void ce_oracle_accel_f32(int n, const double* x, const double* mass, const double* charge,
                         double coulomb_k, double* a);
/* Potential energy (system.cpp:31-41). */
double ce_oracle_pe_f64(int n, const double* x, const double* charge, double coulomb_k);
double ce_oracle_pe_f32(int n, const double* x, const double* charge, double coulomb_k);

/* One explosion from rest: pos0[n][3] -> asymptotic momenta p_out[n][3] = m v
 * after redistribution. Returns the status code. */
int ce_oracle_run_f64(int n, const double* mass, const double* charge, double coulomb_k,
                      const double* pos0, const ce_oracle_cfg* cfg, double* p_out,
                      ce_oracle_stats* st);
int ce_oracle_run_f32(int n, const double* mass, const double* charge, double coulomb_k,
                      const double* pos0, const ce_oracle_cfg* cfg, double* p_out,
                      ce_oracle_stats* st);

/* Batch over S sims, split over host threads (threads <= 0: all online cores).
 * Fixed molecule: n, mass[n], charge[n]; pos [S][n][3]; p_out [S][n][3].
 * Any of steps/status/rejects/ker/t_final/pe_final/ke_before may be NULL. */
void ce_oracle_run_batch(int precision_bits, int n, const double* mass, const double* charge,
                         double coulomb_k, uint64_t S, const double* pos, const ce_oracle_cfg* cfg,
                         double* p_out, uint32_t* steps, uint8_t* status, uint32_t* rejects,
                         double* ker, double* t_final, double* pe_final, double* ke_before,
                         int threads);

/* Mixed molecules: per-sim atom count n_per[S] (2..10), mass/charge [S][10],
 * pos [S][10][3], p_out [S][10][3] (padding rows untouched). */
void ce_oracle_run_batch_mixed(int precision_bits, uint64_t S, const uint8_t* n_per,
                               const double* mass, const double* charge, double coulomb_k,
                               const double* pos, const ce_oracle_cfg* cfg, double* p_out,
                               uint32_t* steps, uint8_t* status, double* ker, int threads);

/* Loose-stop state export for the learned closure's training pairs: runs to
 * pe_stop_fraction (cfg) and returns the raw (un-redistributed) positions and
 * momenta at that point. */
int ce_oracle_run_state_f32(int n, const double* mass, const double* charge, double coulomb_k,
                            const double* pos0, const ce_oracle_cfg* cfg, double* x_out,
                            double* p_out, ce_oracle_stats* st);

#ifdef __cplusplus
}
#endif
#endif /* CE_ORACLE_H */
