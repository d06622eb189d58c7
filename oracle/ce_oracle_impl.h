/*
 * ce_oracle_impl.h -- precision-generic body of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see ce_oracle.h). Included twice by ce_oracle.c,
 * once with REAL=double and once with REAL=float, so one text restates the
 * reference's `Real`-templated scalar engine (include/coulomb/types.hpp:16-20).
 *
 * Required macros: REAL, SFX(name), SQRT, POW, FABS.
 */

/* std::min / std::max semantics (NaN-propagation included): min(a,b) is
 * (b < a) ? b : a and max(a,b) is (a < b) ? b : a. */
#define RMIN(a, b) (((b) < (a)) ? (b) : (a))
#define RMAX(a, b) (((a) < (b)) ? (b) : (a))

/* DP5(4) tableau, src/integrators.cpp:155-167: computed in double and narrowed
 * to Real exactly as the reference's `static constexpr Real` arrays are. */
static const REAL SFX(kA2)[1] = {(REAL)(1.0 / 5)};
static const REAL SFX(kA3)[2] = {(REAL)(3.0 / 40), (REAL)(9.0 / 40)};
static const REAL SFX(kA4)[3] = {(REAL)(44.0 / 45), (REAL)(-56.0 / 15), (REAL)(32.0 / 9)};
static const REAL SFX(kA5)[4] = {(REAL)(19372.0 / 6561), (REAL)(-25360.0 / 2187),
                                 (REAL)(64448.0 / 6561), (REAL)(-212.0 / 729)};
static const REAL SFX(kA6)[5] = {(REAL)(9017.0 / 3168), (REAL)(-355.0 / 33),
                                 (REAL)(46732.0 / 5247), (REAL)(49.0 / 176),
                                 (REAL)(-5103.0 / 18656)};
static const REAL SFX(kA7)[6] = {(REAL)(35.0 / 384),     (REAL)0.0,          (REAL)(500.0 / 1113),
                                 (REAL)(125.0 / 192),    (REAL)(-2187.0 / 6784), (REAL)(11.0 / 84)};
static const REAL* const SFX(kA)[6] = {SFX(kA2), SFX(kA3), SFX(kA4),
                                        SFX(kA5), SFX(kA6), SFX(kA7)};
static const REAL SFX(kE)[7] = {(REAL)(71.0 / 57600),  (REAL)0.0,        (REAL)(-71.0 / 16695),
                                (REAL)(71.0 / 1920),   (REAL)(-17253.0 / 339200),
                                (REAL)(22.0 / 525),    (REAL)(-1.0 / 40)};
/* Controller constants, src/integrators.cpp:169-175. */
#define K_SAFETY ((REAL)0.9)
#define K_MIN_FACTOR ((REAL)0.2)
#define K_MAX_FACTOR ((REAL)10.0)
#define K_EXPONENT ((REAL)(-1.0 / 5.0))
#define K_MAX_REJECTIONS 100

typedef struct SFX(mol) {
  int n;
  REAL mass[CE_ORACLE_NMAX];
  REAL charge[CE_ORACLE_NMAX];
  REAL k;
} SFX(mol);

/* CoulombForce::accelerations, src/system.cpp:5-29 (same operation order). */
static void SFX(accel)(const SFX(mol) * m, REAL (*x)[3], REAL (*a)[3]) {
  const int n = m->n;
  for (int i = 0; i < n; ++i) a[i][0] = a[i][1] = a[i][2] = (REAL)0;
  for (int i = 0; i < n; ++i) {
    for (int j = i + 1; j < n; ++j) {
      const REAL rx = x[i][0] - x[j][0];
      const REAL ry = x[i][1] - x[j][1];
      const REAL rz = x[i][2] - x[j][2];
      const REAL dist2 = rx * rx + ry * ry + rz * rz;
      const REAL inv_dist = (REAL)1 / SQRT(dist2);
      const REAL inv_dist3 = inv_dist / dist2;
      const REAL scale = m->k * m->charge[i] * m->charge[j] * inv_dist3;
      const REAL fx = rx * scale, fy = ry * scale, fz = rz * scale;
      a[i][0] += fx;
      a[i][1] += fy;
      a[i][2] += fz;
      a[j][0] -= fx;
      a[j][1] -= fy;
      a[j][2] -= fz;
    }
  }
  for (int i = 0; i < n; ++i) {
    const REAL inv_m = (REAL)1 / m->mass[i];
    a[i][0] = a[i][0] * inv_m;
    a[i][1] = a[i][1] * inv_m;
    a[i][2] = a[i][2] * inv_m;
  }
}

/* CoulombForce::potential_energy, src/system.cpp:31-41. */
static REAL SFX(pe)(const SFX(mol) * m, REAL (*x)[3]) {
  REAL u = (REAL)0;
  for (int i = 0; i < m->n; ++i) {
    for (int j = i + 1; j < m->n; ++j) {
      const REAL rx = x[i][0] - x[j][0];
      const REAL ry = x[i][1] - x[j][1];
      const REAL rz = x[i][2] - x[j][2];
      u += m->k * m->charge[i] * m->charge[j] / SQRT(rx * rx + ry * ry + rz * rz);
    }
  }
  return u;
}

/* The same potential with every pair term summed in FP64 (CE_ORACLE_FP64 form:
 * the convergence-deciding energy check accumulated in double). */
static double SFX(pe_acc64)(const SFX(mol) * m, REAL (*x)[3]) {
  double u = 0.0;
  for (int i = 0; i < m->n; ++i) {
    for (int j = i + 1; j < m->n; ++j) {
      const REAL rx = x[i][0] - x[j][0];
      const REAL ry = x[i][1] - x[j][1];
      const REAL rz = x[i][2] - x[j][2];
      u += (double)(m->k * m->charge[i] * m->charge[j] / SQRT(rx * rx + ry * ry + rz * rz));
    }
  }
  return u;
}

/* CoulombForce::kinetic_energy, src/system.cpp:43-49. */
static REAL SFX(ke)(const SFX(mol) * m, REAL (*v)[3]) {
  REAL t = (REAL)0;
  for (int i = 0; i < m->n; ++i)
    t += (REAL)0.5 * m->mass[i] * (v[i][0] * v[i][0] + v[i][1] * v[i][1] + v[i][2] * v[i][2]);
  return t;
}

typedef struct SFX(dp45) {
  REAL rtol, atol, h;
  int fsal_valid;
  int kahan;
  REAL kpos[7][CE_ORACLE_NMAX][3]; /* position-derivative stages (stage velocities) */
  REAL kvel[7][CE_ORACLE_NMAX][3]; /* velocity-derivative stages (accelerations)    */
  REAL stage[CE_ORACLE_NMAX][3];   /* scratch positions for force evaluations       */
  REAL probe[CE_ORACLE_NMAX][3];
  REAL cx[CE_ORACLE_NMAX][3], cv[CE_ORACLE_NMAX][3];   /* Kahan compensation (committed) */
  REAL cxn[CE_ORACLE_NMAX][3], cvn[CE_ORACLE_NMAX][3]; /* ... candidate for this attempt */
  uint32_t rejects;
} SFX(dp45);

/* DormandPrince45::err_component, src/integrators.cpp:189-193. */
static REAL SFX(err_component)(const SFX(dp45) * d, REAL err, REAL y_old, REAL y_new) {
  const REAL scale = d->atol + d->rtol * RMAX(FABS(y_old), FABS(y_new));
  const REAL r = err / scale;
  return r * r;
}

/* DormandPrince45::select_initial_step, src/integrators.cpp:197-250. */
static REAL SFX(select_initial_step)(SFX(dp45) * d, const SFX(mol) * m, REAL (*x)[3],
                                     REAL (*v)[3], REAL max_dt) {
  const int n = m->n;
  REAL d0_sq = (REAL)0, d1_sq = (REAL)0;
  for (int i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c) {
      const REAL xc = x[i][c], vc = v[i][c];
      const REAL sx = d->atol + d->rtol * FABS(xc);
      const REAL sv = d->atol + d->rtol * FABS(vc);
      REAL r;
      r = xc / sx;                d0_sq += r * r;
      r = vc / sv;                d0_sq += r * r;
      r = d->kpos[0][i][c] / sx;  d1_sq += r * r;
      r = d->kvel[0][i][c] / sv;  d1_sq += r * r;
    }
  }
  const REAL denom = (REAL)(6 * n);
  const REAL d0 = SQRT(d0_sq / denom);
  const REAL d1 = SQRT(d1_sq / denom);
  const REAL h0 = (d0 < 1e-5 || d1 < 1e-5) ? (REAL)1e-6 : (REAL)0.01 * d0 / d1;

  /* One Euler probe y1 = y0 + h0 f0 for the second-derivative estimate. */
  REAL d2_sq = (REAL)0;
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) d->stage[i][c] = x[i][c] + d->kpos[0][i][c] * h0;
  SFX(accel)(m, d->stage, d->probe);
  for (int i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c) {
      const REAL dv_part = d->kvel[0][i][c] * h0;
      const REAL da_part = d->probe[i][c] - d->kvel[0][i][c];
      const REAL sx = d->atol + d->rtol * FABS(x[i][c]);
      const REAL sv = d->atol + d->rtol * FABS(v[i][c]);
      REAL r;
      r = dv_part / sx; d2_sq += r * r;
      r = da_part / sv; d2_sq += r * r;
    }
  }
  const REAL d2 = SQRT(d2_sq / denom) / h0;
  const REAL h1 = (d1 <= 1e-15 && d2 <= 1e-15) ? RMAX((REAL)1e-6, h0 * (REAL)1e-3)
                                               : POW((REAL)0.01 / RMAX(d1, d2), (REAL)(1.0 / 5.0));
  /* std::min({100*h0, h1, max_dt}): first smallest element. */
  REAL best = 100 * h0;
  if (h1 < best) best = h1;
  if (max_dt < best) best = max_dt;
  return best;
}

/* DormandPrince45::step, src/integrators.cpp:63-147. Returns the step taken, or
 * a negative value once the rejection limit is exceeded (the reference throws
 * std::runtime_error there, src/integrators.cpp:78-82). */
static REAL SFX(step)(SFX(dp45) * d, const SFX(mol) * m, REAL (*x)[3], REAL (*v)[3],
                      REAL max_dt) {
  const int n = m->n;
  if (!d->fsal_valid) {
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c) d->kpos[0][i][c] = v[i][c];
    SFX(accel)(m, x, d->kvel[0]);
    d->fsal_valid = 1;
  }
  if (d->h <= (REAL)0) d->h = SFX(select_initial_step)(d, m, x, v, max_dt);

  int rejected_once = 0;
  for (int attempt = 0;; ++attempt) {
    if (attempt > K_MAX_REJECTIONS) return (REAL)-1;
    const REAL h = RMIN(d->h, max_dt);

    for (int s = 1; s < 7; ++s) {
      const REAL* a = SFX(kA)[s - 1];
      for (int i = 0; i < n; ++i) {
        REAL dx[3] = {0, 0, 0}, dv[3] = {0, 0, 0};
        for (int j = 0; j < s; ++j) {
          const REAL cj = a[j];
          for (int c = 0; c < 3; ++c) {
            dx[c] += d->kpos[j][i][c] * cj;
            dv[c] += d->kvel[j][i][c] * cj;
          }
        }
        for (int c = 0; c < 3; ++c) {
          if (s == 6 && d->kahan) {
            /* Compensated summation of the committed update (no reference
             * counterpart): x_new = x + (dx h - c), c' = (x_new - x) - (dx h - c). */
            const REAL yx = dx[c] * h - d->cx[i][c];
            const REAL tx = x[i][c] + yx;
            d->cxn[i][c] = (tx - x[i][c]) - yx;
            d->stage[i][c] = tx;
            const REAL yv = dv[c] * h - d->cv[i][c];
            const REAL tv = v[i][c] + yv;
            d->cvn[i][c] = (tv - v[i][c]) - yv;
            d->kpos[s][i][c] = tv;
          } else {
            d->stage[i][c] = x[i][c] + dx[c] * h;
            d->kpos[s][i][c] = v[i][c] + dv[c] * h;
          }
        }
      }
      SFX(accel)(m, d->stage, d->kvel[s]);
    }

    REAL err_sq = (REAL)0;
    for (int i = 0; i < n; ++i) {
      REAL ep[3] = {0, 0, 0}, ev[3] = {0, 0, 0};
      for (int s = 0; s < 7; ++s) {
        const REAL cs = SFX(kE)[s];
        for (int c = 0; c < 3; ++c) {
          ep[c] += d->kpos[s][i][c] * cs;
          ev[c] += d->kvel[s][i][c] * cs;
        }
      }
      for (int c = 0; c < 3; ++c) err_sq += SFX(err_component)(d, ep[c] * h, x[i][c], d->stage[i][c]);
      for (int c = 0; c < 3; ++c)
        err_sq += SFX(err_component)(d, ev[c] * h, v[i][c], d->kpos[6][i][c]);
    }
    const REAL error_norm = SQRT(err_sq / (REAL)(6 * n));

    if (error_norm <= (REAL)1) {
      for (int i = 0; i < n; ++i) {
        for (int c = 0; c < 3; ++c) {
          x[i][c] = d->stage[i][c];
          v[i][c] = d->kpos[6][i][c];
          d->kvel[0][i][c] = d->kvel[6][i][c];
          d->kpos[0][i][c] = v[i][c];
          if (d->kahan) {
            d->cx[i][c] = d->cxn[i][c];
            d->cv[i][c] = d->cvn[i][c];
          }
        }
      }
      REAL factor = (error_norm == (REAL)0) ? K_MAX_FACTOR
                                            : RMIN(K_MAX_FACTOR, K_SAFETY * POW(error_norm, K_EXPONENT));
      if (rejected_once) factor = RMIN(factor, (REAL)1);
      d->h = RMIN(h * factor, max_dt);
      return h;
    }
    const REAL factor = RMAX(K_MIN_FACTOR, K_SAFETY * POW(error_norm, K_EXPONENT));
    d->h = h * factor;
    rejected_once = 1;
    d->rejects++;
  }
}

/* VelocityVerlet::step, src/integrators.cpp:16-39: x += v dt + a (0.5 dt dt);
 * a' = a(x); v += (a + a') (0.5 dt); the acceleration is carried between steps. */
typedef struct SFX(vv) {
  int have_accel;
  REAL a[CE_ORACLE_NMAX][3];
} SFX(vv);

static REAL SFX(vv_step)(SFX(vv) * w, const SFX(mol) * m, REAL (*x)[3], REAL (*v)[3], REAL dt) {
  const int n = m->n;
  REAL na[CE_ORACLE_NMAX][3];
  if (!w->have_accel) {
    SFX(accel)(m, x, w->a);
    w->have_accel = 1;
  }
  const REAL h2 = (REAL)0.5 * dt * dt;
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) x[i][c] += v[i][c] * dt + w->a[i][c] * h2;
  SFX(accel)(m, x, na);
  const REAL hd = (REAL)0.5 * dt;
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      v[i][c] += (w->a[i][c] + na[i][c]) * hd;
      w->a[i][c] = na[i][c];
    }
  return dt;
}

static int SFX(all_finite)(int n, REAL (*v)[3]) {
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c)
      if (!isfinite((double)v[i][c])) return 0;
  return 1;
}

/* run_to_convergence, src/driver.cpp:7-46, from rest. p_out gets m v after
 * redistribution; with export_raw the raw x / m v at termination instead. */
static int SFX(run)(int n, const double* mass, const double* charge, double coulomb_k,
                    const double* pos0, const ce_oracle_cfg* cfg, double* p_out, double* x_out,
                    ce_oracle_stats* st, int export_raw) {
  if (n < 1 || n > CE_ORACLE_NMAX) return -1;
  SFX(mol) m;
  m.n = n;
  m.k = (REAL)coulomb_k;
  for (int i = 0; i < n; ++i) {
    m.mass[i] = (REAL)mass[i];
    m.charge[i] = (REAL)charge[i];
  }
  REAL x[CE_ORACLE_NMAX][3], v[CE_ORACLE_NMAX][3];
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      x[i][c] = (REAL)pos0[i * 3 + c];
      v[i][c] = (REAL)0;
    }
  SFX(dp45) d;
  memset(&d, 0, sizeof d);
  d.rtol = (REAL)cfg->rtol;
  d.atol = (REAL)cfg->atol;
  d.kahan = (cfg->mode & CE_ORACLE_KAHAN) != 0;
  const int fp64 = (cfg->mode & CE_ORACLE_FP64) != 0;
  const REAL max_dt = (REAL)cfg->max_dt;

  ce_oracle_stats s;
  memset(&s, 0, sizeof s);
  int status = CE_ORACLE_OK;
  int converged = 0;

  const int verlet = cfg->integrator == 1;
  SFX(vv) w;
  memset(&w, 0, sizeof w);
  if (verlet && cfg->mode != 0) return -1;
  if (!fp64) {
    /* Reference semantics, all in Real. */
    const REAL pe0 = SFX(pe)(&m, x);
    const REAL e0 = pe0 + SFX(ke)(&m, v);
    const REAL pe_stop = (REAL)cfg->pe_stop_fraction * pe0;
    REAL pe = pe0, t = (REAL)0;
    uint64_t steps = 0;
    if (!isfinite((double)pe0)) status = CE_ORACLE_NONFINITE;
    while (status == CE_ORACLE_OK && pe > pe_stop) {
      if (steps >= cfg->max_steps) {
        converged = 0;
        break;
      }
      const REAL dt = verlet ? SFX(vv_step)(&w, &m, x, v, max_dt) : SFX(step)(&d, &m, x, v, max_dt);
      if (dt < (REAL)0) {
        status = CE_ORACLE_REJECT_LIMIT;
        break;
      }
      t += dt;
      ++steps;
      pe = SFX(pe)(&m, x);
      converged = 1;
    }
    s.steps = (uint32_t)steps;
    s.t_final = (double)t;
    s.e0 = (double)e0;
    s.pe_final = (double)pe;
    const REAL ke_before = SFX(ke)(&m, v);
    s.ke_before = (double)ke_before;
    REAL scale = (REAL)1;
    if (!export_raw && cfg->redistribute_energy && ke_before > (REAL)0) {
      scale = SQRT(e0 / ke_before);
      for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) v[i][c] = v[i][c] * scale;
    }
    s.scale = (double)scale;
    s.ke_after = (double)SFX(ke)(&m, v);
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c) {
        p_out[i * 3 + c] = (double)(v[i][c] * m.mass[i]);
        if (x_out) x_out[i * 3 + c] = (double)x[i][c];
      }
    /* A zero-step run (already below pe_stop) is converged, as in the batched
     * engine (include/coulomb/batched_integrator.hpp:138-143). */
    if (steps == 0 && pe <= pe_stop) converged = 1;
  } else {
    /* FP64 time accumulator, FP64-summed potential for the stop test, FP64
     * finalize (batched_integrator.hpp:172-189). */
    const double pe0 = SFX(pe_acc64)(&m, x);
    const double e0 = pe0;
    const double pe_stop = cfg->pe_stop_fraction * pe0;
    double pe = pe0, t = 0.0;
    uint64_t steps = 0;
    if (!isfinite(pe0)) status = CE_ORACLE_NONFINITE;
    while (status == CE_ORACLE_OK && pe > pe_stop) {
      if (steps >= cfg->max_steps) {
        converged = 0;
        break;
      }
      const REAL dt = SFX(step)(&d, &m, x, v, max_dt);
      if (dt < (REAL)0) {
        status = CE_ORACLE_REJECT_LIMIT;
        break;
      }
      t += (double)dt;
      ++steps;
      pe = SFX(pe_acc64)(&m, x);
      converged = 1;
    }
    if (steps == 0 && pe <= pe_stop) converged = 1;
    s.steps = (uint32_t)steps;
    s.t_final = t;
    s.e0 = e0;
    s.pe_final = pe;
    double ke = 0.0;
    for (int i = 0; i < n; ++i) {
      const double vx = v[i][0], vy = v[i][1], vz = v[i][2];
      ke += 0.5 * mass[i] * (vx * vx + vy * vy + vz * vz);
    }
    s.ke_before = ke;
    double scale = 1.0;
    if (!export_raw && cfg->redistribute_energy && ke > 0.0) scale = sqrt(e0 / ke);
    s.scale = scale;
    double ke_after = 0.0;
    for (int i = 0; i < n; ++i) {
      const double mm = mass[i] * scale;
      for (int c = 0; c < 3; ++c) {
        p_out[i * 3 + c] = mm * (double)v[i][c];
        if (x_out) x_out[i * 3 + c] = (double)x[i][c];
        const double vv = (double)v[i][c] * scale;
        ke_after += 0.5 * mass[i] * vv * vv;
      }
    }
    s.ke_after = ke_after;
  }
  s.rejects = d.rejects;
  if (status == CE_ORACLE_OK && !converged) status = CE_ORACLE_MAX_STEPS;
  if (status == CE_ORACLE_OK && !SFX(all_finite)(n, v)) status = CE_ORACLE_NONFINITE;
  s.status = (uint8_t)status;
  if (st) *st = s;
  return status;
}

#undef RMIN
#undef RMAX
#undef K_SAFETY
#undef K_MIN_FACTOR
#undef K_MAX_FACTOR
#undef K_EXPONENT
#undef K_MAX_REJECTIONS
