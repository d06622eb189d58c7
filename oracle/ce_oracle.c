/*
 * ce_oracle.c -- CPU oracle for the batched Coulomb-explosion path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine, loaded by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg, never by the product.
 * Build: oracle/Makefile (no -march, -ffp-contract=off, so float/double
 * arithmetic rounds exactly like the reference scalar engine's SSE2 build).
 */
#include "ce_oracle.h"

#include <math.h>
#include <string.h>

#include <pthread.h>
#include <stdatomic.h>
#include <unistd.h>

#define CE_ORACLE_NMAX 16

/* ---- f64 instantiation (Real = double, the reference's default build) ---- */
#define REAL double
#define SFX(name) name##_f64
#define SQRT sqrt
#define POW pow
#define FABS fabs
#include "ce_oracle_impl.h"
#undef REAL
#undef SFX
#undef SQRT
#undef POW
#undef FABS

/* ---- f32 instantiation (Real = float, COULOMB_SINGLE_PRECISION) ---- */
#define REAL float
#define SFX(name) name##_f32
#define SQRT sqrtf
#define POW powf
#define FABS fabsf
#include "ce_oracle_impl.h"
#undef REAL
#undef SFX
#undef SQRT
#undef POW
#undef FABS

#define DEFINE_PUBLIC(R, S)                                                                      \
  void ce_oracle_accel_##S(int n, const double* x, const double* mass, const double* charge,    \
                           double coulomb_k, double* a) {                                        \
    mol_##S m;                                                                                   \
    R xr[CE_ORACLE_NMAX][3], ar[CE_ORACLE_NMAX][3];                                              \
    if (n < 1 || n > CE_ORACLE_NMAX) return;                                                     \
    m.n = n;                                                                                     \
    m.k = (R)coulomb_k;                                                                          \
    for (int i = 0; i < n; ++i) {                                                                \
      m.mass[i] = (R)mass[i];                                                                    \
      m.charge[i] = (R)charge[i];                                                                \
      for (int c = 0; c < 3; ++c) xr[i][c] = (R)x[i * 3 + c];                                    \
    }                                                                                            \
    accel_##S(&m, xr, ar);                                                                       \
    for (int i = 0; i < n; ++i)                                                                  \
      for (int c = 0; c < 3; ++c) a[i * 3 + c] = (double)ar[i][c];                               \
  }                                                                                              \
  double ce_oracle_pe_##S(int n, const double* x, const double* charge, double coulomb_k) {     \
    mol_##S m;                                                                                   \
    R xr[CE_ORACLE_NMAX][3];                                                                     \
    if (n < 1 || n > CE_ORACLE_NMAX) return NAN;                                                 \
    m.n = n;                                                                                     \
    m.k = (R)coulomb_k;                                                                          \
    for (int i = 0; i < n; ++i) {                                                                \
      m.charge[i] = (R)charge[i];                                                                \
      m.mass[i] = (R)1;                                                                          \
      for (int c = 0; c < 3; ++c) xr[i][c] = (R)x[i * 3 + c];                                    \
    }                                                                                            \
    return (double)pe_##S(&m, xr);                                                               \
  }                                                                                              \
  int ce_oracle_run_##S(int n, const double* mass, const double* charge, double coulomb_k,      \
                        const double* pos0, const ce_oracle_cfg* cfg, double* p_out,             \
                        ce_oracle_stats* st) {                                                   \
    return run_##S(n, mass, charge, coulomb_k, pos0, cfg, p_out, NULL, st, 0);                   \
  }

DEFINE_PUBLIC(double, f64)
DEFINE_PUBLIC(float, f32)

int ce_oracle_run_state_f32(int n, const double* mass, const double* charge, double coulomb_k,
                            const double* pos0, const ce_oracle_cfg* cfg, double* x_out,
                            double* p_out, ce_oracle_stats* st) {
  return run_f32(n, mass, charge, coulomb_k, pos0, cfg, p_out, x_out, st, 1);
}

static void run_one(int precision_bits, int n, const double* mass, const double* charge,
                    double coulomb_k, const double* pos, const ce_oracle_cfg* cfg, double* p,
                    ce_oracle_stats* st) {
  if (precision_bits == 32)
    run_f32(n, mass, charge, coulomb_k, pos, cfg, p, NULL, st, 0);
  else
    run_f64(n, mass, charge, coulomb_k, pos, cfg, p, NULL, st, 0);
}

static double ker_of(int n, const double* mass, const double* p) {
  double k = 0.0;
  for (int i = 0; i < n; ++i) {
    const double px = p[i * 3], py = p[i * 3 + 1], pz = p[i * 3 + 2];
    k += (px * px + py * py + pz * pz) / (2.0 * mass[i]);
  }
  return k;
}

/* Work split over host threads: a shared atomic cursor hands out blocks of 16
 * sims, so uneven per-sim step counts balance across threads. */
typedef struct batch_job {
  int precision_bits, n, mixed;
  const uint8_t* n_per;
  const double *mass, *charge, *pos;
  double coulomb_k;
  uint64_t S;
  const ce_oracle_cfg* cfg;
  double* p_out;
  uint32_t *steps, *rejects;
  uint8_t* status;
  double *ker, *t_final, *pe_final, *ke_before;
  _Atomic uint64_t cursor;
} batch_job;

static void do_sim(batch_job* j, uint64_t s) {
  ce_oracle_stats st;
  int n;
  const double *m, *q, *x;
  double* p;
  if (j->mixed) {
    n = j->n_per[s];
    m = j->mass + s * 10;
    q = j->charge + s * 10;
    x = j->pos + s * 30;
    p = j->p_out + s * 30;
  } else {
    n = j->n;
    m = j->mass;
    q = j->charge;
    x = j->pos + s * (uint64_t)n * 3;
    p = j->p_out + s * (uint64_t)n * 3;
  }
  run_one(j->precision_bits, n, m, q, j->coulomb_k, x, j->cfg, p, &st);
  if (j->steps) j->steps[s] = st.steps;
  if (j->status) j->status[s] = st.status;
  if (j->rejects) j->rejects[s] = st.rejects;
  if (j->ker) j->ker[s] = ker_of(n, m, p);
  if (j->t_final) j->t_final[s] = st.t_final;
  if (j->pe_final) j->pe_final[s] = st.pe_final;
  if (j->ke_before) j->ke_before[s] = st.ke_before;
}

static void* batch_worker(void* arg) {
  batch_job* j = (batch_job*)arg;
  for (;;) {
    const uint64_t s0 = atomic_fetch_add(&j->cursor, 16);
    if (s0 >= j->S) break;
    const uint64_t s1 = s0 + 16 < j->S ? s0 + 16 : j->S;
    for (uint64_t s = s0; s < s1; ++s) do_sim(j, s);
  }
  return NULL;
}

static void run_job(batch_job* j, int threads) {
  if (threads <= 0) {
    const long nc = sysconf(_SC_NPROCESSORS_ONLN);
    threads = nc > 0 ? (int)nc : 1;
  }
  if (threads > 256) threads = 256;
  atomic_store(&j->cursor, 0);
  if (threads == 1) {
    batch_worker(j);
    return;
  }
  pthread_t tid[256];
  int started = 0;
  for (int t = 0; t < threads; ++t)
    if (pthread_create(&tid[t], NULL, batch_worker, j) == 0) ++started;
  if (started == 0) batch_worker(j);
  for (int t = 0; t < started; ++t) pthread_join(tid[t], NULL);
}

void ce_oracle_run_batch(int precision_bits, int n, const double* mass, const double* charge,
                         double coulomb_k, uint64_t S, const double* pos, const ce_oracle_cfg* cfg,
                         double* p_out, uint32_t* steps, uint8_t* status, uint32_t* rejects,
                         double* ker, double* t_final, double* pe_final, double* ke_before,
                         int threads) {
  batch_job j;
  memset(&j, 0, sizeof j);
  j.precision_bits = precision_bits;
  j.n = n;
  j.mass = mass;
  j.charge = charge;
  j.pos = pos;
  j.coulomb_k = coulomb_k;
  j.S = S;
  j.cfg = cfg;
  j.p_out = p_out;
  j.steps = steps;
  j.status = status;
  j.rejects = rejects;
  j.ker = ker;
  j.t_final = t_final;
  j.pe_final = pe_final;
  j.ke_before = ke_before;
  run_job(&j, threads);
}

void ce_oracle_run_batch_mixed(int precision_bits, uint64_t S, const uint8_t* n_per,
                               const double* mass, const double* charge, double coulomb_k,
                               const double* pos, const ce_oracle_cfg* cfg, double* p_out,
                               uint32_t* steps, uint8_t* status, double* ker, int threads) {
  batch_job j;
  memset(&j, 0, sizeof j);
  j.precision_bits = precision_bits;
  j.mixed = 1;
  j.n_per = n_per;
  j.mass = mass;
  j.charge = charge;
  j.pos = pos;
  j.coulomb_k = coulomb_k;
  j.S = S;
  j.cfg = cfg;
  j.p_out = p_out;
  j.steps = steps;
  j.status = status;
  j.ker = ker;
  run_job(&j, threads);
}
