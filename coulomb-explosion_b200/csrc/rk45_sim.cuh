// rk45_sim.cuh -- one Coulomb explosion per thread, entirely in registers.
//
// Device-side restatement of the reference's per-sim integration:
//   pair force / potential         src/system.cpp:5-41, include/coulomb/batched_force.hpp:31-110
//   DP5(4) attempt + controller    src/integrators.cpp:63-147
//   Hairer initial step            src/integrators.cpp:197-250
//   stop test + redistribution     src/driver.cpp:7-46, FP64 finalize as in
//                                  include/coulomb/batched_integrator.hpp:172-189
// B200 choices (not in the reference): each thread owns one simulation (no
// shared-dt lockstep, batched_integrator.hpp:10-16), pair terms use the MUFU
// rsqrt plus FMAs, stages are stored as accelerations only (dp45_tableau.cuh),
// the potential energy for the stop test is fused into the stage-7 force
// evaluation (x_7 is x_new, FSAL), and because every simulation starts at rest
// the Hairer Euler probe has x_1 = x_0 exactly, so its force evaluation equals
// k1 and is not recomputed.
#pragma once

#include <cstdint>
#include <type_traits>

#include "ce_gpu.h"
#include "dp45_tableau.cuh"

namespace ce {

// Per-molecule constants for the fixed-molecule path, passed as a kernel
// parameter so every use is a constant-bank operand.
struct FixedMol {
  float pc[CE_MAX_ATOMS * CE_MAX_ATOMS];  // k q_i q_j, row-major [i*N + j], narrowed from double
  float inv_m[CE_MAX_ATOMS];              // 1 / m_i (float)
  double mass[CE_MAX_ATOMS];              // m_i (double, FP64 finalize)
  float q[CE_MAX_ATOMS];                  // q_i (lane-per-atom layout: pair constant q_i * (k q_j))
  float kq[CE_MAX_ATOMS];                 // k q_i
  float k;                                // Coulomb constant narrowed to float (the reference's Real k_)
};

struct RunParams {
  const float* pos;  // [S][N][3]
  float* momenta;    // [S][N][3]
  double* ker;
  uint32_t* steps;
  uint8_t* status;
  uint32_t* rejects;
  double* t_final;
  double* pe_final;
  double* ke_before;
  float* positions;  // [S][N][3] positions at termination (optional)
  double* e0;        // [S] initial energy (optional)
  unsigned long long* cursor;  // work-queue head (device scratch, zeroed per launch)
  unsigned long long S;
  float rtol, atol, max_dt;
  float pe_stop_f;   // pe_stop_fraction as float (FP32 stop test: Real * Real)
  double pe_stop_d;  // pe_stop_fraction as double (FP64 stop test)
  uint32_t max_steps;
  int32_t redistribute;
  int32_t refill_threshold;
  int32_t skip_empty;  // mixed batches: rows with n_atoms == 0 are left untouched (no outputs written)
};

template <int N, int MODE>
struct Sim {
  static constexpr bool kKahan = (MODE & CE_PREC_KAHAN) != 0;
  static constexpr bool kF64 = (MODE & CE_PREC_FP64) != 0;
  static constexpr int KC = kKahan ? N : 1;
  using Acc = typename std::conditional<kF64, double, float>::type;

  float x[N][3];
  float v[N][3];
  float k[6][N][3];  // k[0] = a(x) (FSAL), k[1..5] = stage accelerations 2..6
  float cx[KC][3];   // Kahan compensation of the committed x / v updates
  float cv[KC][3];
  float h;
  Acc t;
  Acc e0;
  Acc pe_stop;
  uint32_t steps, rejects, rej_in_step;
  bool rej_once;
  unsigned long long sim;
};

// a_i = (1/m_i) sum_j k q_i q_j r_ij / |r_ij|^3 with Newton's third law, and
// (if WITH_PE) pe += sum_{i<j} k q_i q_j / |r_ij|.
template <int N, bool WITH_PE, typename TPE>
__device__ __forceinline__ void pair_forces(const float (&x)[N][3], float (&a)[N][3],
                                            const FixedMol& M, TPE& pe) {
#pragma unroll
  for (int i = 0; i < N; ++i) a[i][0] = a[i][1] = a[i][2] = 0.0f;
#pragma unroll
  for (int i = 0; i < N; ++i) {
#pragma unroll
    for (int j = i + 1; j < N; ++j) {
      const float rx = x[i][0] - x[j][0];
      const float ry = x[i][1] - x[j][1];
      const float rz = x[i][2] - x[j][2];
      const float d2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
      const float rinv = rsqrtf(d2);
      const float u = M.pc[i * N + j] * rinv;  // pair potential k q_i q_j / r
      if (WITH_PE) pe += static_cast<TPE>(u);
      const float s = u * (rinv * rinv);       // k q_i q_j / r^3
      a[i][0] = fmaf(rx, s, a[i][0]);
      a[i][1] = fmaf(ry, s, a[i][1]);
      a[i][2] = fmaf(rz, s, a[i][2]);
      a[j][0] = fmaf(-rx, s, a[j][0]);
      a[j][1] = fmaf(-ry, s, a[j][1]);
      a[j][2] = fmaf(-rz, s, a[j][2]);
    }
  }
#pragma unroll
  for (int i = 0; i < N; ++i) {
    a[i][0] *= M.inv_m[i];
    a[i][1] *= M.inv_m[i];
    a[i][2] *= M.inv_m[i];
  }
}

// FP64 finalize: KE, s = sqrt(E0/KE), p_i = (m_i s) v_i, KER; then the per-sim
// output record. A converged sim with non-finite momenta is CE_SIM_NONFINITE.
template <int N, int MODE>
__device__ __forceinline__ void finalize(const Sim<N, MODE>& s, int status, double pe_final,
                                         const RunParams& P, const FixedMol& M) {
  double ke = 0.0;
  bool finite = true;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const double vx = s.v[i][0], vy = s.v[i][1], vz = s.v[i][2];
    ke += 0.5 * M.mass[i] * (vx * vx + vy * vy + vz * vz);
    finite = finite && isfinite(vx) && isfinite(vy) && isfinite(vz);
  }
  if (status == CE_SIM_OK && !finite) status = CE_SIM_NONFINITE;
  const double sc = (P.redistribute && ke > 0.0) ? sqrt(static_cast<double>(s.e0) / ke) : 1.0;
  double ker = 0.0;
  float* dst = P.momenta + s.sim * (3ull * N);
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const double mm = M.mass[i] * sc;
    const double px = mm * static_cast<double>(s.v[i][0]);
    const double py = mm * static_cast<double>(s.v[i][1]);
    const double pz = mm * static_cast<double>(s.v[i][2]);
    dst[i * 3 + 0] = static_cast<float>(px);
    dst[i * 3 + 1] = static_cast<float>(py);
    dst[i * 3 + 2] = static_cast<float>(pz);
    ker += (px * px + py * py + pz * pz) / (2.0 * M.mass[i]);
  }
  if (P.ker) P.ker[s.sim] = ker;
  if (P.steps) P.steps[s.sim] = s.steps;
  if (P.status) P.status[s.sim] = static_cast<uint8_t>(status);
  if (P.rejects) P.rejects[s.sim] = s.rejects;
  if (P.t_final) P.t_final[s.sim] = static_cast<double>(s.t);
  if (P.pe_final) P.pe_final[s.sim] = pe_final;
  if (P.ke_before) P.ke_before[s.sim] = ke;
  if (P.e0) P.e0[s.sim] = static_cast<double>(s.e0);
  if (P.positions) {
    float* xp = P.positions + s.sim * (3ull * N);
#pragma unroll
    for (int i = 0; i < N; ++i) {
      xp[i * 3 + 0] = s.x[i][0];
      xp[i * 3 + 1] = s.x[i][1];
      xp[i * 3 + 2] = s.x[i][2];
    }
  }
}

// Hairer's initial step from rest (src/integrators.cpp:197-250 with v0 = 0:
// every velocity term is 0, sv = atol, and the probe accelerations equal k1).
template <int N, int MODE>
__device__ __forceinline__ float initial_step(const Sim<N, MODE>& s, const RunParams& P) {
  float d0_sq = 0.0f, d1_sq = 0.0f, d2_sq = 0.0f;
#pragma unroll
  for (int i = 0; i < N; ++i) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float sx = P.atol + P.rtol * fabsf(s.x[i][c]);
      const float r0 = s.x[i][c] / sx;
      const float r1 = s.k[0][i][c] / P.atol;
      d0_sq += r0 * r0;
      d1_sq += r1 * r1;
    }
  }
  const float denom = static_cast<float>(6 * N);
  const float d0 = sqrtf(d0_sq / denom);
  const float d1 = sqrtf(d1_sq / denom);
  const float h0 = (static_cast<double>(d0) < 1e-5 || static_cast<double>(d1) < 1e-5)
                       ? 1e-6f
                       : 0.01f * d0 / d1;
#pragma unroll
  for (int i = 0; i < N; ++i) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float sx = P.atol + P.rtol * fabsf(s.x[i][c]);
      const float r = (s.k[0][i][c] * h0) / sx;  // (v1 - v0) / sx; (a1 - a0) = 0
      d2_sq += r * r;
    }
  }
  const float d2 = sqrtf(d2_sq / denom) / h0;
  const float h1 = (static_cast<double>(d1) <= 1e-15 && static_cast<double>(d2) <= 1e-15)
                       ? fmaxf(1e-6f, h0 * 1e-3f)
                       : powf(0.01f / fmaxf(d1, d2), 0.2f);
  float hmin = 100.0f * h0;
  if (h1 < hmin) hmin = h1;
  if (P.max_dt < hmin) hmin = P.max_dt;
  return hmin;
}

// Load sim `sim` and prepare its first step. Returns false when the sim is
// already finished (written out) and the lane stays idle.
template <int N, int MODE>
__device__ __forceinline__ bool init_sim(Sim<N, MODE>& s, unsigned long long sim,
                                         const RunParams& P, const FixedMol& M) {
  using Acc = typename Sim<N, MODE>::Acc;
  s.sim = sim;
  const float* src = P.pos + sim * (3ull * N);
#pragma unroll
  for (int i = 0; i < N; ++i) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      s.x[i][c] = __ldg(src + i * 3 + c);
      s.v[i][c] = 0.0f;
    }
  }
#pragma unroll
  for (int i = 0; i < Sim<N, MODE>::KC; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) s.cx[i][c] = s.cv[i][c] = 0.0f;
  Acc pe0 = Acc(0);
  pair_forces<N, true>(s.x, s.k[0], M, pe0);
  s.t = Acc(0);
  s.steps = 0;
  s.rejects = 0;
  s.rej_in_step = 0;
  s.rej_once = false;
  s.e0 = pe0;  // E_0 = PE_0 + KE_0, KE_0 = 0 (batched_integrator.hpp:137)
  if (Sim<N, MODE>::kF64)
    s.pe_stop = static_cast<Acc>(P.pe_stop_d * static_cast<double>(pe0));
  else
    s.pe_stop = static_cast<Acc>(P.pe_stop_f * static_cast<float>(pe0));
  if (!isfinite(static_cast<double>(pe0))) {
    finalize(s, CE_SIM_NONFINITE, static_cast<double>(pe0), P, M);
    return false;
  }
  if (!(pe0 > s.pe_stop)) {  // already at or below the stop (driver.cpp:19)
    finalize(s, CE_SIM_OK, static_cast<double>(pe0), P, M);
    return false;
  }
  if (P.max_steps == 0u) {
    finalize(s, CE_SIM_MAX_STEPS, static_cast<double>(pe0), P, M);
    return false;
  }
  s.h = initial_step(s, P);
  return true;
}

// One DP5(4) attempt (src/integrators.cpp:83-146) plus, on acceptance, the
// driver's stop test (src/driver.cpp:19-30). Returns false once the sim is
// finished and written out.
template <int N, int MODE>
__device__ __forceinline__ bool attempt(Sim<N, MODE>& s, const RunParams& P, const FixedMol& M) {
  using S = Sim<N, MODE>;
  using Acc = typename S::Acc;
  const float hh = (P.max_dt < s.h) ? P.max_dt : s.h;  // std::min(h_, max_dt)

  // Stages 2..6: x_s = x + h (c_s v + h sum_l abar_sl k_l); k_s = a(x_s).
  {
    float xs[N][3];
#pragma unroll
    for (int si = 1; si <= 5; ++si) {
#pragma unroll
      for (int i = 0; i < N; ++i) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float sum = 0.0f;
#pragma unroll
          for (int l = 0; l + 1 < si; ++l) sum = fmaf(c_abar[si + 1][l + 1], s.k[l][i][c], sum);
          const float inner = fmaf(hh, sum, c_c[si + 1] * s.v[i][c]);
          xs[i][c] = fmaf(hh, inner, s.x[i][c]);
        }
      }
      Acc unused = Acc(0);
      pair_forces<N, false>(xs, s.k[si], M, unused);
    }
  }

  // Stage 7 (row = 5th-order weights): x_new, v_new, the position half of the
  // error and the k1..k6 part of the velocity error, before k7 is known.
  float xn[N][3], vn[N][3], evp[N][3];
  float cxn[S::KC][3], cvn[S::KC][3];
  float err_sq = 0.0f;
#pragma unroll
  for (int i = 0; i < N; ++i) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float sx = 0.0f, sv = 0.0f, se = 0.0f, sev = 0.0f;
#pragma unroll
      for (int l = 0; l < 6; ++l) {
        if (l < 5) sx = fmaf(c_abar[7][l + 1], s.k[l][i][c], sx);
        if (l != 1) sv = fmaf(c_b[l + 1], s.k[l][i][c], sv);  // b_2 = 0
        se = fmaf(c_ebar[l + 1], s.k[l][i][c], se);
        if (l != 1) sev = fmaf(c_e[l + 1], s.k[l][i][c], sev);  // E_2 = 0
      }
      const float incx = hh * fmaf(hh, sx, s.v[i][c]);  // c_7 = 1
      const float incv = hh * sv;
      if (S::kKahan) {
        const float yx = incx - s.cx[i][c];
        xn[i][c] = s.x[i][c] + yx;
        cxn[i][c] = (xn[i][c] - s.x[i][c]) - yx;
        const float yv = incv - s.cv[i][c];
        vn[i][c] = s.v[i][c] + yv;
        cvn[i][c] = (vn[i][c] - s.v[i][c]) - yv;
      } else {
        xn[i][c] = s.x[i][c] + incx;
        vn[i][c] = s.v[i][c] + incv;
      }
      evp[i][c] = sev;
      const float ex = (hh * hh) * se;
      const float scx = fmaf(P.rtol, fmaxf(fabsf(s.x[i][c]), fabsf(xn[i][c])), P.atol);
      const float r = __fdividef(ex, scx);
      err_sq = fmaf(r, r, err_sq);
    }
  }
  float k7[N][3];
  Acc pe_new = Acc(0);
  pair_forces<N, true>(xn, k7, M, pe_new);
#pragma unroll
  for (int i = 0; i < N; ++i) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float ev = hh * fmaf(c_e[7], k7[i][c], evp[i][c]);
      const float scv = fmaf(P.rtol, fmaxf(fabsf(s.v[i][c]), fabsf(vn[i][c])), P.atol);
      const float r = __fdividef(ev, scv);
      err_sq = fmaf(r, r, err_sq);
    }
  }
  const float en = sqrtf(err_sq * (1.0f / static_cast<float>(6 * N)));

  if (en <= 1.0f) {
#pragma unroll
    for (int i = 0; i < N; ++i) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        s.x[i][c] = xn[i][c];
        s.v[i][c] = vn[i][c];
        s.k[0][i][c] = k7[i][c];
        if (S::kKahan) {
          s.cx[i][c] = cxn[i][c];
          s.cv[i][c] = cvn[i][c];
        }
      }
    }
    float factor = (en == 0.0f) ? kMaxFactor : fminf(kMaxFactor, kSafety * __powf(en, kExponent));
    if (s.rej_once) factor = fminf(factor, 1.0f);
    const float hn = hh * factor;
    s.h = (P.max_dt < hn) ? P.max_dt : hn;
    s.t += static_cast<Acc>(hh);
    s.steps += 1u;
    s.rej_in_step = 0;
    s.rej_once = false;
    if (!(pe_new > s.pe_stop)) {
      finalize(s, CE_SIM_OK, static_cast<double>(pe_new), P, M);
      return false;
    }
    if (s.steps >= P.max_steps) {
      finalize(s, CE_SIM_MAX_STEPS, static_cast<double>(pe_new), P, M);
      return false;
    }
    return true;
  }
  const float factor = fmaxf(kMinFactor, kSafety * __powf(en, kExponent));
  s.h = hh * factor;
  s.rej_once = true;
  s.rejects += 1u;
  s.rej_in_step += 1u;
  if (s.rej_in_step > static_cast<uint32_t>(kMaxRejections)) {
    finalize(s, CE_SIM_REJECT_LIMIT, static_cast<double>(pe_new), P, M);
    return false;
  }
  return true;
}

// Persistent kernel: each warp keeps its 32 lanes busy by pulling sim indices
// from a global cursor (one warp-aggregated atomicAdd per refill) whenever at
// least `refill_threshold` lanes are idle; no lane waits on another lane's sim.
template <int N, int MODE>
__global__ void __launch_bounds__(256) rk45_fixed_kernel(const RunParams P, const FixedMol M) {
  Sim<N, MODE> s;
  bool active = false;
  bool queue_empty = false;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    if (!queue_empty && idle != 0u &&
        (idle == 0xffffffffu || __popc(idle) >= P.refill_threshold)) {
      const int cnt = __popc(idle);
      const int leader = __ffs(idle) - 1;
      unsigned long long base = 0ull;
      if (static_cast<int>(lane) == leader) base = atomicAdd(P.cursor, static_cast<unsigned long long>(cnt));
      base = __shfl_sync(0xffffffffu, base, leader);
      queue_empty = (base + static_cast<unsigned long long>(cnt) >= P.S);
      if (!active) {
        const unsigned long long sim = base + static_cast<unsigned long long>(__popc(idle & lt_mask));
        if (sim < P.S) active = init_sim(s, sim, P, M);
      }
    }
    if (!__any_sync(0xffffffffu, active)) {
      if (queue_empty) break;
      continue;
    }
    if (active) active = attempt(s, P, M);
  }
}

using FixedKernelFn = void (*)(RunParams, FixedMol);
// One dispatch function per precision mode, defined in kernels_fixed.cu.
FixedKernelFn fixed_kernel_m0(int n);
FixedKernelFn fixed_kernel_m1(int n);
FixedKernelFn fixed_kernel_m2(int n);
FixedKernelFn fixed_kernel_m3(int n);

}  // namespace ce
