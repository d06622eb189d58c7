// rk45_atom.cuh -- lane-per-atom layout: one simulation per group of N lanes.
//
// Same integration as rk45_sim.cuh (src/integrators.cpp:63-250,
// src/driver.cpp:7-46, FP64 finalize as batched_integrator.hpp:172-189) with a
// different mapping: lane (g, i) of a warp owns atom i of the g-th simulation in
// that warp, G = 32 / N simulations per warp. Each lane keeps only its atom's
// x, v and six stage accelerations (~3x fewer registers than a whole sim per
// thread), so occupancy is high and N = 10 needs no spills.
//
// Per force evaluation a lane publishes (x, y, z, k q_i) to its slot of a
// per-warp shared-memory buffer (double-buffered, one __syncwarp per
// evaluation) and reads its N-1 partners with 16-byte loads; the partner set is
// fixed per lane, so there is no self pair. The pair term is computed twice
// (once on each side) instead of using Newton's third law. Sums over a
// simulation (error norm, potential, kinetic energy, Hairer norms) are
// gathered with N shuffles in a fixed order, so every lane of a group holds the
// bit-identical value and takes the same accept/reject and stop decisions.
//
// Control flow is warp-uniform: every lane executes every attempt (lanes whose
// simulation is finished, or that carry no atom, compute on stale data and
// commit nothing), which keeps the shared-memory exchange fully synchronised.
// The six stage force evaluations share one copy of the code (rolled stage
// loop, coefficients from constant memory), which keeps the hot loop small.
#pragma once

#include <cstdint>
#include <type_traits>

#include "ce_gpu.h"
#include "dp45_tableau.cuh"
#include "rk45_sim.cuh"

namespace ce {

template <int N>
struct AtomShape {
  static constexpr int G = 32 / N;     // simulations per warp
  static constexpr int USED = G * N;   // lanes carrying an atom
};

struct AtomConsts {
  float qi;      // q_i (pair constant = q_i * (k q_j))
  float kqi;     // k q_i, published with the position
  float inv_m;   // 1 / m_i
  double mass;   // m_i
};

// Fixed-order sum over the N lanes [base, base + N) of a group; every lane of
// the group returns the identical value.
template <int N, typename T>
__device__ __forceinline__ T gsum(T v, int base) {
  T s = __shfl_sync(0xffffffffu, v, base);
#pragma unroll
  for (int j = 1; j < N; ++j) s += __shfl_sync(0xffffffffu, v, base + j);
  return s;
}

template <int N, int MODE>
struct AtomLane {
  static constexpr bool kKahan = (MODE & CE_PREC_KAHAN) != 0;
  static constexpr bool kF64 = (MODE & CE_PREC_FP64) != 0;
  using Acc = typename std::conditional<kF64, double, float>::type;
  float x[3], v[3];
  float k[6][3];
  float cx[3], cv[3];
  float h;
  Acc t, e0, pe_stop;
  uint32_t steps, rejects, rej_in_step;
  bool rej_once;
  unsigned long long sim;
};

// One force evaluation for every lane of the warp: publish (xs, kq_i), read the
// N-1 partners, accumulate a_i and (optionally) this lane's half of the pair
// potential. `slot` is this lane's buffer index, `nbr[d]` the partners'.
template <int N, typename Acc>
__device__ __forceinline__ void lane_force(float4* __restrict__ buf, int& par, int slot, const int (&nbr)[N - 1],
                                           const float (&xs)[3], const AtomConsts& ac, bool want_pe,
                                           float (&a)[3], Acc& pe_half) {
  float4* b = buf + par * 32;
  par ^= 1;
  b[slot] = make_float4(xs[0], xs[1], xs[2], ac.kqi);
  __syncwarp();
  float ax = 0.0f, ay = 0.0f, az = 0.0f;
  Acc pe = Acc(0);
#pragma unroll
  for (int d = 0; d < N - 1; ++d) {
    const float4 o = b[nbr[d]];
    const float rx = xs[0] - o.x;
    const float ry = xs[1] - o.y;
    const float rz = xs[2] - o.z;
    const float d2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
    const float rinv = rsqrtf(d2);
    const float u = (ac.qi * o.w) * rinv;  // k q_i q_j / r
    if (want_pe) pe += static_cast<Acc>(u);
    const float s = u * (rinv * rinv);
    ax = fmaf(rx, s, ax);
    ay = fmaf(ry, s, ay);
    az = fmaf(rz, s, az);
  }
  a[0] = ax * ac.inv_m;
  a[1] = ay * ac.inv_m;
  a[2] = az * ac.inv_m;
  pe_half = pe;
}

// FP64 finalize, executed by every lane of the warp (the reductions are full-warp
// shuffles); lanes with status < 0 compute but write nothing. Each finishing
// lane writes its atom's momentum, lane i = 0 of the group the per-sim scalars.
template <int N, int MODE>
__device__ __forceinline__ void atom_finalize(const AtomLane<N, MODE>& s, int status, double pe_final,
                                              const AtomConsts& ac, int ai, int base, const RunParams& P) {
  const double vx = s.v[0], vy = s.v[1], vz = s.v[2];
  const double ke = gsum<N>(0.5 * ac.mass * (vx * vx + vy * vy + vz * vz), base);
  const int fin = gsum<N>((isfinite(vx) && isfinite(vy) && isfinite(vz)) ? 0 : 1, base);
  if (status == CE_SIM_OK && fin != 0) status = CE_SIM_NONFINITE;
  const double sc = (P.redistribute && ke > 0.0) ? sqrt(static_cast<double>(s.e0) / ke) : 1.0;
  const double mm = ac.mass * sc;
  const double px = mm * vx, py = mm * vy, pz = mm * vz;
  const double ker = gsum<N>((px * px + py * py + pz * pz) / (2.0 * ac.mass), base);
  if (status < 0) return;
  float* dst = P.momenta + s.sim * (3ull * N) + 3 * ai;
  dst[0] = static_cast<float>(px);
  dst[1] = static_cast<float>(py);
  dst[2] = static_cast<float>(pz);
  if (ai == 0) {
    if (P.ker) P.ker[s.sim] = ker;
    if (P.steps) P.steps[s.sim] = s.steps;
    if (P.status) P.status[s.sim] = static_cast<uint8_t>(status);
    if (P.rejects) P.rejects[s.sim] = s.rejects;
    if (P.t_final) P.t_final[s.sim] = static_cast<double>(s.t);
    if (P.pe_final) P.pe_final[s.sim] = pe_final;
    if (P.ke_before) P.ke_before[s.sim] = ke;
  }
}

// Persistent lane-per-atom kernel for one fixed molecule. Block = 32 * W
// threads; each warp owns 2 x 32 float4 of shared memory.
template <int N, int MODE>
__global__ void __launch_bounds__(256) rk45_atom_kernel(const RunParams P, const FixedMol M) {
  using L = AtomLane<N, MODE>;
  using Acc = typename L::Acc;
  constexpr int G = AtomShape<N>::G;
  constexpr int USED = AtomShape<N>::USED;
  extern __shared__ float4 smem_pos[];
  float4* buf = smem_pos + (threadIdx.x >> 5) * 64;
  const int lane = static_cast<int>(threadIdx.x & 31u);
  const bool has_atom = lane < USED;
  const int g = has_atom ? lane / N : G;  // idle lanes form their own (empty) group
  const int ai = has_atom ? lane - g * N : 0;
  const int base = has_atom ? g * N : lane;
  const bool leader = has_atom && ai == 0;
  int nbr[N - 1];
#pragma unroll
  for (int d = 0; d < N - 1; ++d) {
    int j = ai + 1 + d;
    if (j >= N) j -= N;
    nbr[d] = has_atom ? base + j : lane;
  }
  AtomConsts ac;
  ac.qi = M.q[ai];
  ac.kqi = M.kq[ai];
  ac.inv_m = M.inv_m[ai];
  ac.mass = M.mass[ai];
  L s;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    s.x[c] = s.v[c] = s.cx[c] = s.cv[c] = 0.0f;
#pragma unroll
    for (int l = 0; l < 6; ++l) s.k[l][c] = 0.0f;
  }
  s.h = 0.0f;
  s.t = s.e0 = s.pe_stop = Acc(0);
  s.steps = s.rejects = s.rej_in_step = 0u;
  s.rej_once = false;
  s.sim = 0ull;
  int par = 0;
  bool active = false;
  bool queue_empty = false;
  const unsigned lt_mask = (1u << lane) - 1u;

  for (;;) {
    // ---- refill: one claim per idle group, warp-aggregated ----
    bool fresh = false;
    const unsigned idle = __ballot_sync(0xffffffffu, leader && !active);
    if (!queue_empty && idle != 0u &&
        (__popc(idle) >= P.refill_threshold || __ballot_sync(0xffffffffu, active) == 0u)) {
      const int cnt = __popc(idle);
      const int first = __ffs(idle) - 1;
      unsigned long long b0 = 0ull;
      if (lane == first) b0 = atomicAdd(P.cursor, static_cast<unsigned long long>(cnt));
      b0 = __shfl_sync(0xffffffffu, b0, first);
      queue_empty = (b0 + static_cast<unsigned long long>(cnt) >= P.S);
      unsigned long long mine = ~0ull;
      if (leader && !active) mine = b0 + static_cast<unsigned long long>(__popc(idle & lt_mask));
      mine = __shfl_sync(0xffffffffu, mine, base);
      if (has_atom && !active && mine < P.S) {
        fresh = true;
        s.sim = mine;
      }
    }
    // ---- init of freshly claimed sims (all lanes take part in the exchange) ----
    if (__ballot_sync(0xffffffffu, fresh) != 0u) {
      int fin_st = -1;
      if (fresh) {
        const float* src = P.pos + s.sim * (3ull * N) + 3 * ai;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          s.x[c] = __ldg(src + c);
          s.v[c] = 0.0f;
          s.cx[c] = s.cv[c] = 0.0f;
        }
      }
      float a0[3];
      Acc peh;
      lane_force<N, Acc>(buf, par, lane, nbr, s.x, ac, true, a0, peh);
      const Acc pe0 = gsum<N>(peh, base) * Acc(0.5);
      // Hairer norms from rest (sv = atol, probe accelerations = k1).
      float d0p = 0.0f, d1p = 0.0f;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float sx = P.atol + P.rtol * fabsf(s.x[c]);
        const float r0 = s.x[c] / sx;
        const float r1 = a0[c] / P.atol;
        d0p += r0 * r0;
        d1p += r1 * r1;
      }
      const float d0sq = gsum<N>(d0p, base), d1sq = gsum<N>(d1p, base);
      const float denom = static_cast<float>(6 * N);
      const float d0 = sqrtf(d0sq / denom), d1 = sqrtf(d1sq / denom);
      const float h0 = (static_cast<double>(d0) < 1e-5 || static_cast<double>(d1) < 1e-5) ? 1e-6f : 0.01f * d0 / d1;
      float d2p = 0.0f;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float sx = P.atol + P.rtol * fabsf(s.x[c]);
        const float r = (a0[c] * h0) / sx;
        d2p += r * r;
      }
      const float d2 = sqrtf(gsum<N>(d2p, base) / denom) / h0;
      if (fresh) {
#pragma unroll
        for (int c = 0; c < 3; ++c) s.k[0][c] = a0[c];
        const float h1 = (static_cast<double>(d1) <= 1e-15 && static_cast<double>(d2) <= 1e-15)
                             ? fmaxf(1e-6f, h0 * 1e-3f)
                             : powf(0.01f / fmaxf(d1, d2), 0.2f);
        float hm = 100.0f * h0;
        if (h1 < hm) hm = h1;
        if (P.max_dt < hm) hm = P.max_dt;
        s.h = hm;
        s.t = Acc(0);
        s.steps = s.rejects = s.rej_in_step = 0u;
        s.rej_once = false;
        s.e0 = pe0;
        if (L::kF64)
          s.pe_stop = static_cast<Acc>(P.pe_stop_d * static_cast<double>(pe0));
        else
          s.pe_stop = static_cast<Acc>(P.pe_stop_f * static_cast<float>(pe0));
        active = true;
        if (!isfinite(static_cast<double>(pe0))) fin_st = CE_SIM_NONFINITE;
        else if (!(pe0 > s.pe_stop)) fin_st = CE_SIM_OK;
        else if (P.max_steps == 0u) fin_st = CE_SIM_MAX_STEPS;
        if (fin_st >= 0) active = false;
      }
      if (__ballot_sync(0xffffffffu, fin_st >= 0) != 0u)
        atom_finalize<N, MODE>(s, fin_st, static_cast<double>(pe0), ac, ai, base, P);
    }
    if (__ballot_sync(0xffffffffu, active) == 0u) {
      if (queue_empty) break;
      continue;
    }

    // ---- one DP5(4) attempt, all lanes ----
    const float hh = (P.max_dt < s.h) ? P.max_dt : s.h;
    float xs[3], a[3];
    float cxn[3] = {0.0f, 0.0f, 0.0f};
    Acc pe_half = Acc(0);
#pragma unroll 1
    for (int si = 1; si <= 6; ++si) {
      const float cs = c_c[si + 1];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float sum = 0.0f;
#pragma unroll
        for (int l = 0; l < 5; ++l)
          if (l + 1 < si) sum = fmaf(c_abar[si + 1][l + 1], s.k[l][c], sum);
        const float inc = hh * fmaf(hh, sum, cs * s.v[c]);
        if (L::kKahan && si == 6) {
          const float y = inc - s.cx[c];
          xs[c] = s.x[c] + y;
          cxn[c] = (xs[c] - s.x[c]) - y;
        } else {
          xs[c] = s.x[c] + inc;
        }
      }
      lane_force<N, Acc>(buf, par, lane, nbr, xs, ac, si == 6, a, pe_half);
      switch (si) {
        case 1: s.k[1][0] = a[0]; s.k[1][1] = a[1]; s.k[1][2] = a[2]; break;
        case 2: s.k[2][0] = a[0]; s.k[2][1] = a[1]; s.k[2][2] = a[2]; break;
        case 3: s.k[3][0] = a[0]; s.k[3][1] = a[1]; s.k[3][2] = a[2]; break;
        case 4: s.k[4][0] = a[0]; s.k[4][1] = a[1]; s.k[4][2] = a[2]; break;
        case 5: s.k[5][0] = a[0]; s.k[5][1] = a[1]; s.k[5][2] = a[2]; break;
        default: break;
      }
    }
    // Stage 7 done: xs = x_new, a = k7. Velocity update and error estimate.
    float vn[3], cvn[3] = {0.0f, 0.0f, 0.0f};
    float errp = 0.0f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float sv = 0.0f, se = 0.0f, sev = 0.0f;
#pragma unroll
      for (int l = 0; l < 6; ++l) {
        if (l != 1) sv = fmaf(c_b[l + 1], s.k[l][c], sv);
        se = fmaf(c_ebar[l + 1], s.k[l][c], se);
        if (l != 1) sev = fmaf(c_e[l + 1], s.k[l][c], sev);
      }
      const float incv = hh * sv;
      if (L::kKahan) {
        const float y = incv - s.cv[c];
        vn[c] = s.v[c] + y;
        cvn[c] = (vn[c] - s.v[c]) - y;
      } else {
        vn[c] = s.v[c] + incv;
      }
      const float ex = (hh * hh) * se;
      const float ev = hh * fmaf(c_e[7], a[c], sev);
      const float scx = fmaf(P.rtol, fmaxf(fabsf(s.x[c]), fabsf(xs[c])), P.atol);
      const float scv = fmaf(P.rtol, fmaxf(fabsf(s.v[c]), fabsf(vn[c])), P.atol);
      const float rx = __fdividef(ex, scx);
      const float rv = __fdividef(ev, scv);
      errp = fmaf(rx, rx, errp);
      errp = fmaf(rv, rv, errp);
    }
    const float err_sq = gsum<N>(errp, base);
    const Acc pe_new = gsum<N>(pe_half, base) * Acc(0.5);
    int fin_st = -1;
    if (active) {
      const float en = sqrtf(err_sq * (1.0f / static_cast<float>(6 * N)));
      if (en <= 1.0f) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          s.x[c] = xs[c];
          s.v[c] = vn[c];
          s.k[0][c] = a[c];
          if (L::kKahan) {
            s.cx[c] = cxn[c];
            s.cv[c] = cvn[c];
          }
        }
        float factor = (en == 0.0f) ? kMaxFactor : fminf(kMaxFactor, kSafety * __powf(en, kExponent));
        if (s.rej_once) factor = fminf(factor, 1.0f);
        const float hn = hh * factor;
        s.h = (P.max_dt < hn) ? P.max_dt : hn;
        s.t += static_cast<Acc>(hh);
        s.steps += 1u;
        s.rej_in_step = 0u;
        s.rej_once = false;
        if (!(pe_new > s.pe_stop)) fin_st = CE_SIM_OK;
        else if (s.steps >= P.max_steps) fin_st = CE_SIM_MAX_STEPS;
      } else {
        const float factor = fmaxf(kMinFactor, kSafety * __powf(en, kExponent));
        s.h = hh * factor;
        s.rej_once = true;
        s.rejects += 1u;
        s.rej_in_step += 1u;
        if (s.rej_in_step > static_cast<uint32_t>(kMaxRejections)) fin_st = CE_SIM_REJECT_LIMIT;
      }
      if (fin_st >= 0) active = false;
    }
    if (__ballot_sync(0xffffffffu, fin_st >= 0) != 0u)
      atom_finalize<N, MODE>(s, fin_st, static_cast<double>(pe_new), ac, ai, base, P);
  }
}

using AtomKernelFn = void (*)(RunParams, FixedMol);
AtomKernelFn atom_kernel_m0(int n);
AtomKernelFn atom_kernel_m1(int n);
AtomKernelFn atom_kernel_m2(int n);
AtomKernelFn atom_kernel_m3(int n);

}  // namespace ce
