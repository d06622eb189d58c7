// rk45_atom.cuh -- lane-per-atom layout: one simulation per group of N lanes.
//
// Same integration as rk45_sim.cuh (src/integrators.cpp:63-250,
// src/driver.cpp:7-46, FP64 finalize as batched_integrator.hpp:172-189) with a
// different mapping: lane (g, i) of a warp owns atom i of the g-th simulation in
// that warp, G = 32 / N simulations per warp. Each lane keeps only its atom's
// x, v and six stage accelerations (~3x fewer registers than a whole sim per
// thread), so occupancy is high and N = 10 needs no spills.
//
// Per force evaluation a lane reads its partners' positions from their lanes
// with register shuffles; the partner set is fixed per lane, so there is no
// self pair, and the lane's pair constants k q_i q_j sit in registers. Each pair
// term is evaluated by one lane of the pair and handed to the other with
// shuffles (Newton's third law, see lane_force). Sums over a simulation (error
// norm, potential, kinetic energy, Hairer norms) are gathered with N shuffles in
// a fixed order, so every lane of a group holds the bit-identical value and
// takes the same accept/reject and stop decisions.
//
// Control flow is warp-uniform: every lane executes every attempt (lanes whose
// simulation is finished, or that carry no atom, compute on stale data and
// commit nothing), which keeps the full-warp shuffles of the exchange valid.
// The stage loop is unrolled: a lane carries three components, so the six
// force loops stay small and every coefficient is a compile-time operand.
//
// One warp loop (atom_loop<N, MODE, MIXED, STATE>) serves three kernels:
//   rk45_atom_kernel<N, MODE>    one fixed molecule (include/ce_gpu.h ce_run*)
//   rk45_mixed_kernel<MODE>      mixed 2..10-atom molecules, one persistent
//                                launch walking the size buckets 10 -> 2
//   rk45_bucket_kernel<N, MODE>  one size bucket (the per-size launch schedule)
#pragma once

#include <cstdint>
#include <type_traits>

#include "ce_gpu.h"
#include "dp45_tableau.cuh"
#include "rk45_sim.cuh"

namespace ce {

// Largest block of the lane-per-atom kernels. Declaring it as the launch bound
// lets the register allocator size for 128-thread blocks (N = 5: 92 registers,
// 5 blocks per SM) instead of for 256-thread ones (80 registers with spills, so
// that 3 such blocks fit), which ran CH4 ~3 % slower.
constexpr int kAtomMaxBlock = 128;

// Default refill granularity: with G = 32 / n sims per warp in the lane-per-atom
// layout, a warp refills once floor((G - 1) / 3) of its groups are idle, at
// least one (measured: CH4, G = 6: 1 beats 2 and 3 by 0.5 % and 1.5 %; stiff
// H2O, G = 10: 3 beats 2 and 4 by 0.3 % and 3.7 %; N = 10, G = 3: 1).
// Thread-per-sim refills once 4 of a warp's 32 sims are idle (CH4: 4 beats 1,
// 2, 6 and 8 by 0.2 to 6 %), two threads per sim once 2 of its 16 are; a
// single atom finishes at once, so 1. A refill threshold of 0 in RunParams or
// ce_tuning means this per-size default.
__host__ __device__ constexpr int default_refill(int n, int lanes_per_sim) {
  return n < 2 ? 1
               : (lanes_per_sim < 2 ? 4
                                    : ((lanes_per_sim == 2 && n >= 3)
                                           ? 2
                                           : ((32 / n - 1) / 3 > 1 ? (32 / n - 1) / 3 : 1)));
}

// Default layout of a fixed-molecule run (ce_tuning::lanes_per_sim): one thread
// per sim for up to kThreadMaxAtoms atoms (with Kahan compensation, whose terms
// take four more stage slots, from 4 atoms up), two threads per sim from 7
// atoms (with Kahan compensation for even counts only), otherwise one lane per
// atom. Measured at the tight point, 1e6 sims, explosions/s:
//   CH4, plain FP32: thread 2.78e8, lane 2.15e8; full precision form (Kahan +
//   FP64 t/E): thread 2.13e8, lane 2.02e8. Stiff H2O plain: thread 5.22e8,
//   lane 4.66e8; full precision: thread 4.24e8, lane 4.32e8.
//   Random 7 / 8 / 9 / 10-atom molecules (q in 1..3), plain: two-thread 1.14e8 /
//   1.08e8 / 7.27e7 / 6.99e7, lane 1.13e8 / 9.60e7 / 6.85e7 / 5.90e7, thread
//   (7 and 10) 1.13e8 / 4.21e7; full precision: two-thread 1.03e8 / 9.78e7 /
//   5.87e7 / 5.61e7, lane 1.05e8 / 9.12e7 / 6.54e7 / 5.54e7. C2H6-like plain:
//   two-thread 7.49e7, lane 6.34e7.
constexpr int kThreadMaxAtoms = 6;
__host__ __device__ constexpr int default_lanes(int n, int mode) {
  return n < 2 ? 1
               : (n <= kThreadMaxAtoms ? (((mode & CE_PREC_KAHAN) == 0 || n >= 4) ? 1 : n)
                                       : (((mode & CE_PREC_KAHAN) == 0 || n % 2 == 0) ? 2 : n));
}

// Layout of a fixed-molecule run from ce_tuning::lanes_per_sim: 1 = one thread
// per sim, 2 = two threads per sim (3 or more atoms; with 2 atoms that is one
// lane per atom), anything larger = one lane per atom.
enum : int { kLayoutThread = 0, kLayoutPair = 1, kLayoutAtom = 2 };
__host__ __device__ constexpr int layout_of(int n, int lanes_per_sim) {
  return (lanes_per_sim <= 1 || n < 2) ? kLayoutThread
                                       : ((lanes_per_sim == 2 && n >= 3) ? kLayoutPair : kLayoutAtom);
}

// Threads per block, dynamic shared memory and sims per block of a
// fixed-molecule launch in layout `layout` (atom_block: the lane-per-atom
// kernel's block size; the other two kernels fix theirs at compile time).
struct FixedLaunchShape {
  int block;
  size_t smem;
  unsigned long long sims_per_block;
};
inline FixedLaunchShape fixed_launch_shape(int n, int layout, int mode, int atom_block) {
  if (layout == kLayoutThread) {
    const int b = thread_block(n);
    return {b, thread_smem_bytes(n, b, mode), static_cast<unsigned long long>(b)};
  }
  if (layout == kLayoutPair) return {kPairBlock, pair_smem_bytes(n, mode), static_cast<unsigned long long>(kPairBlock / 2)};
  const int b = atom_block < kAtomMaxBlock ? atom_block : kAtomMaxBlock;
  return {b, 0, static_cast<unsigned long long>(b / 32) * static_cast<unsigned long long>(32 / n)};
}

template <int N>
struct AtomShape {
  static constexpr int G = 32 / N;     // simulations per warp
  static constexpr int USED = G * N;   // lanes carrying an atom
};

struct AtomConsts {
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

// A lane's 3-vector as an (x, y) pair plus z, so component-wise arithmetic
// runs on the packed FP32x2 instructions (one FFMA2 / FADD2 / FMUL2 for x and
// y). Every packed operation rounds each element exactly like its scalar
// counterpart (a - b is evaluated as fma(-1, b, a), which is exact), so the
// results equal the scalar formulation bit for bit.
struct V3 {
  float2 xy;
  float z;
  __device__ __forceinline__ float get(int c) const { return c == 0 ? xy.x : (c == 1 ? xy.y : z); }
};
__device__ __forceinline__ V3 v3_zero() { return {make_float2(0.0f, 0.0f), 0.0f}; }
// s * a + c
__device__ __forceinline__ V3 v3_fma(float s, const V3& a, const V3& c) {
  return {__ffma2_rn(bcast(s), a.xy, c.xy), fmaf(s, a.z, c.z)};
}
__device__ __forceinline__ V3 v3_mul(float s, const V3& a) { return {__fmul2_rn(bcast(s), a.xy), s * a.z}; }
__device__ __forceinline__ V3 v3_add(const V3& a, const V3& b) { return {__fadd2_rn(a.xy, b.xy), a.z + b.z}; }
__device__ __forceinline__ V3 v3_sub(const V3& a, const V3& b) {
  return {__ffma2_rn(bcast(-1.0f), b.xy, a.xy), a.z - b.z};
}

template <int N, int MODE>
struct AtomLane {
  static constexpr bool kKahan = (MODE & CE_PREC_KAHAN) != 0;
  static constexpr bool kF64 = (MODE & CE_PREC_FP64) != 0;
  using Acc = typename std::conditional<kF64, double, float>::type;
  V3 x, v;
  V3 k[6];
  V3 cx, cv;
  float h;
  Acc t, e0, pe_stop;
  uint32_t steps, rejects, rej_in_step;
  bool rej_once;
  unsigned long long sim;
};

// One force evaluation for every lane of the warp: read the partners'
// positions from their lanes with register shuffles, accumulate a_i and
// (optionally) this lane's share of the potential. Every lane of the warp takes
// part (the shuffles are full-warp), so no shared memory or __syncwarp is
// involved; a shuffle costs one shared-memory-pipe wavefront, against four
// (plus bank conflicts where a group wraps) for a 16-byte shared-memory read.
//
// Newton's third law across lanes: partner d of lane i is atom i+1+d (mod N).
// Lane i evaluates the pair terms f_d = k q_i q_j r / |r|^3 (r = x_i - x_j) for
// d < H = (N-1)/2 only, adds them to its own acceleration, and receives -f from
// the lane that evaluated its pair as that lane's d-th term (lane i-1-d) with
// one shuffle per component. For even N the opposite atom (d = N/2 - 1) pairs
// two lanes symmetrically; both evaluate it, each taking half of its potential.
// Every pair's potential is counted once: the group sum of pe_part is PE.
template <int N, typename Acc>
__device__ __forceinline__ void lane_force(const int (&nbr)[N - 1], const int (&recv)[N - 1],
                                           const float (&pcv)[N - 1], const V3& xs, const AtomConsts& ac,
                                           bool want_pe, V3& a, Acc& pe_part) {
  constexpr int H = (N - 1) / 2;
  constexpr bool kOpp = (N % 2) == 0;
  float2 axy = make_float2(0.0f, 0.0f);
  float az = 0.0f;
  float2 fxy[H > 0 ? H : 1];
  float fz[H > 0 ? H : 1];
  Acc pe = Acc(0);
#pragma unroll
  for (int d = 0; d < H; ++d) {
    const float ox = __shfl_sync(0xffffffffu, xs.xy.x, nbr[d]);
    const float oy = __shfl_sync(0xffffffffu, xs.xy.y, nbr[d]);
    const float oz = __shfl_sync(0xffffffffu, xs.z, nbr[d]);
    const float2 rxy = __ffma2_rn(bcast(-1.0f), make_float2(ox, oy), xs.xy);
    const float rz = xs.z - oz;
    const float d2 = fmaf(rxy.x, rxy.x, fmaf(rxy.y, rxy.y, rz * rz));
    const float rinv = rsqrtf(d2);
    const float u = pcv[d] * rinv;  // k q_i q_j / r
    if (want_pe) pe += static_cast<Acc>(u);
    const float sc = u * (rinv * rinv);
    fxy[d] = __fmul2_rn(rxy, bcast(sc));
    fz[d] = rz * sc;
    axy = __fadd2_rn(axy, fxy[d]);
    az += fz[d];
  }
  if (kOpp) {
    constexpr int d = N / 2 - 1;
    const float ox = __shfl_sync(0xffffffffu, xs.xy.x, nbr[d]);
    const float oy = __shfl_sync(0xffffffffu, xs.xy.y, nbr[d]);
    const float oz = __shfl_sync(0xffffffffu, xs.z, nbr[d]);
    const float2 rxy = __ffma2_rn(bcast(-1.0f), make_float2(ox, oy), xs.xy);
    const float rz = xs.z - oz;
    const float d2 = fmaf(rxy.x, rxy.x, fmaf(rxy.y, rxy.y, rz * rz));
    const float rinv = rsqrtf(d2);
    const float u = pcv[d] * rinv;
    if (want_pe) pe += static_cast<Acc>(0.5f * u);
    const float sc = u * (rinv * rinv);
    axy = __ffma2_rn(rxy, bcast(sc), axy);
    az = fmaf(rz, sc, az);
  }
#pragma unroll
  for (int d = 0; d < H; ++d) {
    const float gx = __shfl_sync(0xffffffffu, fxy[d].x, recv[d]);
    const float gy = __shfl_sync(0xffffffffu, fxy[d].y, recv[d]);
    axy = __ffma2_rn(bcast(-1.0f), make_float2(gx, gy), axy);
    az -= __shfl_sync(0xffffffffu, fz[d], recv[d]);
  }
  a.xy = __fmul2_rn(axy, bcast(ac.inv_m));
  a.z = az * ac.inv_m;
  pe_part = pe;
}

// FP64 finalize, executed by every lane of the warp (the reductions are full-warp
// shuffles); lanes with status < 0 compute but write nothing. Each finishing
// lane writes its atom's momentum, lane i = 0 of the group the per-sim scalars.
template <int N, int MODE, int STRIDE, bool STATE>
__device__ __forceinline__ void atom_finalize(const AtomLane<N, MODE>& s, int status, double pe_final,
                                              const AtomConsts& ac, int ai, int base, const RunParams& P) {
  const double vx = s.v.xy.x, vy = s.v.xy.y, vz = s.v.z;
  const double ke = gsum<N>(0.5 * ac.mass * (vx * vx + vy * vy + vz * vz), base);
  // Non-finite velocity anywhere in the group: one vote, masked to the group's lanes.
  const unsigned bad = __ballot_sync(0xffffffffu, !(isfinite(vx) && isfinite(vy) && isfinite(vz)));
  const unsigned gmask = ((1u << N) - 1u) << base;
  if (status == CE_SIM_OK && (bad & gmask) != 0u) status = CE_SIM_NONFINITE;
  // s = sqrt(E0 / KE), formed as E0 rsqrt(E0 KE) (one reciprocal square root
  // instead of a division and a square root) when E0 > 0.
  const double e0d = static_cast<double>(s.e0);
  const double sc =
      (P.redistribute && ke > 0.0) ? (e0d > 0.0 ? e0d * rsqrt(e0d * ke) : sqrt(e0d / ke)) : 1.0;
  const double mm = ac.mass * sc;
  const double px = mm * vx, py = mm * vy, pz = mm * vz;
  // KER = sum |p_i|^2 / (2 m_i) with p_i = s m_i v_i, i.e. s^2 KE (the FP64
  // group sum above), so no per-atom division or second group sum is needed.
  const double ker = (sc * sc) * ke;
  if (status < 0) return;
  float* dst = P.momenta + s.sim * (3ull * STRIDE) + 3 * ai;
  dst[0] = static_cast<float>(px);
  dst[1] = static_cast<float>(py);
  dst[2] = static_cast<float>(pz);
  if (P.positions) {
    float* xp = P.positions + s.sim * (3ull * STRIDE) + 3 * ai;
    xp[0] = s.x.xy.x;
    xp[1] = s.x.xy.y;
    xp[2] = s.x.z;
  }
  if (ai == 0 && P.e0) P.e0[s.sim] = static_cast<double>(s.e0);
  if (STATE && P.save_h) {  // the integrator state this sim stopped in (a resumable run's input)
    const unsigned long long row = s.sim * (3ull * STRIDE) + 3 * ai;
    P.save_pos[row] = s.x.xy.x;
    P.save_pos[row + 1] = s.x.xy.y;
    P.save_pos[row + 2] = s.x.z;
    P.save_vel[row] = s.v.xy.x;
    P.save_vel[row + 1] = s.v.xy.y;
    P.save_vel[row + 2] = s.v.z;
    if (AtomLane<N, MODE>::kKahan && P.save_comp) {
      float* c = P.save_comp + s.sim * (6ull * STRIDE) + 6 * ai;
      c[0] = s.cx.xy.x;
      c[1] = s.cx.xy.y;
      c[2] = s.cx.z;
      c[3] = s.cv.xy.x;
      c[4] = s.cv.xy.y;
      c[5] = s.cv.z;
    }
    if (ai == 0) {
      P.save_h[s.sim] = status == CE_SIM_OK ? s.h : 0.0f;
      P.save_t[s.sim] = static_cast<double>(s.t);
      P.save_steps[s.sim] = s.steps;
      P.save_rejects[s.sim] = s.rejects;
      P.save_e0[s.sim] = static_cast<double>(s.e0);
    }
  }
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

// The warp loop: keep this warp's G groups busy with sims of exactly N atoms
// drawn from one work queue (cursor over [0, count), mapped through perm when
// non-null) until the queue is empty and every group has finished. MIXED reads
// each sim's masses and charges from X; otherwise the fixed molecule M.
template <int N, int MODE, bool MIXED, bool STATE>
__device__ __forceinline__ void atom_loop(const RunParams& P, const FixedMol& M, const MixedIn& X,
                                          unsigned long long* cursor, unsigned long long count,
                                          const uint32_t* perm, int refill) {
  using L = AtomLane<N, MODE>;
  using Acc = typename L::Acc;
  constexpr int G = AtomShape<N>::G;
  constexpr int USED = AtomShape<N>::USED;
  constexpr int STRIDE = MIXED ? kMixedStride : N;
  const int lane = static_cast<int>(threadIdx.x & 31u);
  const bool has_atom = lane < USED;
  const int g = has_atom ? lane / N : G;  // idle lanes form their own (empty) group
  const int ai = has_atom ? lane - g * N : 0;
  const int base = has_atom ? g * N : lane;
  const bool leader = has_atom && ai == 0;
  int nbr[N - 1];
  int recv[N - 1];  // lane that evaluates this lane's pair as its d-th term
  int pidx[N - 1];  // partner atom index j for each d
#pragma unroll
  for (int d = 0; d < N - 1; ++d) {
    int j = ai + 1 + d;
    if (j >= N) j -= N;
    pidx[d] = j;
    nbr[d] = has_atom ? base + j : lane;
    int r = ai - 1 - d;
    if (r < 0) r += N;
    recv[d] = has_atom ? base + r : lane;
  }
  AtomConsts ac;
  float pcv[N - 1];
  if (!MIXED) {
    ac.inv_m = M.inv_m[ai];
    ac.mass = M.mass[ai];
#pragma unroll
    for (int d = 0; d < N - 1; ++d) pcv[d] = M.pc[ai * N + pidx[d]];
  } else {
    ac.inv_m = 1.0f;
    ac.mass = 1.0;
#pragma unroll
    for (int d = 0; d < N - 1; ++d) pcv[d] = 0.0f;
  }
  L s;
  s.x = s.v = s.cx = s.cv = v3_zero();
#pragma unroll
  for (int l = 0; l < 6; ++l) s.k[l] = v3_zero();
  s.h = 0.0f;
  s.t = s.e0 = s.pe_stop = Acc(0);
  s.steps = s.rejects = s.rej_in_step = 0u;
  s.rej_once = false;
  s.sim = 0ull;
  bool active = false;
  bool queue_empty = count == 0ull;
  const unsigned lt_mask = (1u << lane) - 1u;

  // A group whose sim stopped is written out at the warp's next refill (or once
  // the queue is empty): the finalize is a whole-warp step, so the groups that
  // stopped since the last refill share one. Until then the group's rejection
  // counter and stop threshold, no longer needed, hold the status and the final
  // potential energy.
  bool pending = false;
  for (;;) {
    // ---- refill: one claim per idle group, warp-aggregated ----
    bool fresh = false;
    const unsigned idle = __ballot_sync(0xffffffffu, leader && !active);
    const bool claim = !queue_empty && idle != 0u && (__popc(idle) >= refill || __ballot_sync(0xffffffffu, active) == 0u);
    if ((claim || queue_empty) && __ballot_sync(0xffffffffu, pending) != 0u) {
      atom_finalize<N, MODE, STRIDE, STATE>(s, pending ? static_cast<int>(s.rej_in_step) : -1,
                                            static_cast<double>(s.pe_stop), ac, ai, base, P);
      pending = false;
    }
    if (claim) {
      const int cnt = __popc(idle);
      const int first = __ffs(idle) - 1;
      unsigned long long b0 = 0ull;
      if (lane == first) b0 = atomicAdd(cursor, static_cast<unsigned long long>(cnt));
      b0 = __shfl_sync(0xffffffffu, b0, first);
      queue_empty = (b0 + static_cast<unsigned long long>(cnt) >= count);
      unsigned long long mine = ~0ull;
      if (leader && !active) mine = b0 + static_cast<unsigned long long>(__popc(idle & lt_mask));
      mine = __shfl_sync(0xffffffffu, mine, base);
      if (has_atom && !active && mine < count) {
        fresh = true;
        s.sim = perm ? static_cast<unsigned long long>(perm[mine]) : mine;
      }
    }
    // ---- init of freshly claimed sims (all lanes take part in the exchange) ----
    if (__ballot_sync(0xffffffffu, fresh) != 0u) {
      int fin_st = -1;
      bool resumed = false;  // continue from a saved state (res_h > 0) instead of from rest
      if (fresh) {
        if (STATE && P.res_h) resumed = __ldg(P.res_h + s.sim) > 0.0f;
        const unsigned long long row = s.sim * (3ull * STRIDE) + 3 * ai;
        const float* src = (resumed ? P.res_pos : P.pos) + row;
        s.x = {make_float2(__ldg(src), __ldg(src + 1)), __ldg(src + 2)};
        s.v = s.cx = s.cv = v3_zero();
        if (resumed) {
          s.v = {make_float2(__ldg(P.res_vel + row), __ldg(P.res_vel + row + 1)), __ldg(P.res_vel + row + 2)};
          if (L::kKahan) {
            const float* c = P.res_comp + s.sim * (6ull * STRIDE) + 6 * ai;
            s.cx = {make_float2(__ldg(c), __ldg(c + 1)), __ldg(c + 2)};
            s.cv = {make_float2(__ldg(c + 3), __ldg(c + 4)), __ldg(c + 5)};
          }
        }
      }
      if (MIXED) {
        // This sim's constants: pair constants (k q_i) q_j formed in double and
        // narrowed, as the fixed path does (batched_integrator.hpp:79-87).
        double qi = 0.0, mi = 1.0;
        if (fresh) {
          qi = __ldg(X.charge + s.sim * kMixedStride + ai);
          mi = __ldg(X.mass + s.sim * kMixedStride + ai);
        }
#pragma unroll
        for (int d = 0; d < N - 1; ++d) {
          const double qj = __shfl_sync(0xffffffffu, qi, nbr[d]);
          if (fresh) pcv[d] = static_cast<float>(X.coulomb_k * qi * qj);
        }
        if (fresh) {
          ac.mass = mi;
          ac.inv_m = static_cast<float>(1.0 / mi);
        }
      }
      V3 a0;
      Acc peh;
      lane_force<N, Acc>(nbr, recv, pcv, s.x, ac, true, a0, peh);
      const Acc pe0 = gsum<N>(peh, base);
      // Hairer norms from rest (sv = atol, probe accelerations = k1). The
      // initial step is a heuristic (any h within the controller's reach gives
      // the same converged answer), so its quotients use the fast forms.
      const float inv_atol = __frcp_rn(P.atol);
      float d0p = 0.0f, d1p = 0.0f;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float sx = P.atol + P.rtol * fabsf(s.x.get(c));
        const float r0 = __fdividef(s.x.get(c), sx);
        const float r1 = a0.get(c) * inv_atol;
        d0p += r0 * r0;
        d1p += r1 * r1;
      }
      constexpr float inv_denom = 1.0f / static_cast<float>(6 * N);
      const float d0 = sqrt_approx(gsum<N>(d0p, base) * inv_denom);
      const float d1 = sqrt_approx(gsum<N>(d1p, base) * inv_denom);
      const float h0 = (static_cast<double>(d0) < 1e-5 || static_cast<double>(d1) < 1e-5)
                           ? 1e-6f
                           : __fdividef(0.01f * d0, d1);
      float d2p = 0.0f;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float sx = P.atol + P.rtol * fabsf(s.x.get(c));
        const float r = __fdividef(a0.get(c) * h0, sx);
        d2p += r * r;
      }
      const float d2 = __fdividef(sqrt_approx(gsum<N>(d2p, base) * inv_denom), h0);
      if (STATE && fresh && resumed) {
        // The saved state follows an accepted step: k1 = a(x) is bit for bit the
        // k7 of that step, and the driver's stop test runs again on the current
        // potential (src/driver.cpp:19-30), as the uninterrupted run would.
        s.k[0] = a0;
        s.h = __ldg(P.res_h + s.sim);
        s.t = static_cast<Acc>(P.res_t[s.sim]);
        s.steps = P.res_steps[s.sim];
        s.rejects = P.res_rejects[s.sim];
        s.rej_in_step = 0u;
        s.rej_once = false;
        s.e0 = static_cast<Acc>(P.res_e0[s.sim]);
        if (L::kF64)
          s.pe_stop = static_cast<Acc>(P.pe_stop_d * static_cast<double>(s.e0));
        else
          s.pe_stop = static_cast<Acc>(P.pe_stop_f * static_cast<float>(s.e0));
        active = true;
        if (!(pe0 > s.pe_stop)) fin_st = CE_SIM_OK;
        else if (s.steps >= P.max_steps) fin_st = CE_SIM_MAX_STEPS;
        if (fin_st >= 0) active = false;
      } else if (fresh) {
        s.k[0] = a0;
        const float h1 = (static_cast<double>(d1) <= 1e-15 && static_cast<double>(d2) <= 1e-15)
                             ? fmaxf(1e-6f, h0 * 1e-3f)
                             : __powf(__fdividef(0.01f, fmaxf(d1, d2)), 0.2f);
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
        atom_finalize<N, MODE, STRIDE, STATE>(s, fin_st, static_cast<double>(pe0), ac, ai, base, P);
    }
    if (__ballot_sync(0xffffffffu, active) == 0u) {
      if (queue_empty) break;
      continue;
    }

    // ---- one DP5(4) attempt, all lanes ----
    const float hh = (P.max_dt < s.h) ? P.max_dt : s.h;
    const float hh2 = hh * hh;
    const V3 hv = v3_mul(hh, s.v);
    V3 xs, a;
    V3 cxn = v3_zero();
    Acc pe_half = Acc(0);
#pragma unroll
    for (int si = 1; si <= 6; ++si) {
      // x_s = x + c_s h v + h^2 sum_l abar_sl k_l (stage 2 has no k term).
      V3 inc = v3_mul(c_c[si + 1], hv);
      if (si > 1) {
        V3 sum = v3_mul(c_abar[si + 1][1], s.k[0]);
#pragma unroll
        for (int l = 1; l + 1 < si; ++l) sum = v3_fma(c_abar[si + 1][l + 1], s.k[l], sum);
        inc = v3_fma(hh2, sum, inc);
      }
      if (L::kKahan && si == 6) {
        const V3 y = v3_sub(inc, s.cx);
        xs = v3_add(s.x, y);
        cxn = v3_sub(v3_sub(xs, s.x), y);
      } else {
        xs = v3_add(s.x, inc);
      }
      lane_force<N, Acc>(nbr, recv, pcv, xs, ac, si == 6, a, pe_half);
      if (si <= 5) s.k[si] = a;
    }
    // Stage 7 done: xs = x_new, a = k7. Velocity update and error estimate.
    V3 sv = v3_zero(), se = v3_zero(), sev = v3_zero();
#pragma unroll
    for (int l = 0; l < 6; ++l) {
      if (l != 1) sv = v3_fma(c_b[l + 1], s.k[l], sv);
      se = v3_fma(c_ebar[l + 1], s.k[l], se);
      if (l != 1) sev = v3_fma(c_e[l + 1], s.k[l], sev);
    }
    const V3 incv = v3_mul(hh, sv);
    V3 vn, cvn = v3_zero();
    if (L::kKahan) {
      const V3 y = v3_sub(incv, s.cv);
      vn = v3_add(s.v, y);
      cvn = v3_sub(v3_sub(vn, s.v), y);
    } else {
      vn = v3_add(s.v, incv);
    }
    const V3 ex = v3_mul(hh2, se);
    const V3 ev = v3_mul(hh, v3_fma(c_e[7], a, sev));
    // Scaled errors e / (atol + rtol max(|y0|, |y1|)); x and y packed.
    const float2 scx = __ffma2_rn(bcast(P.rtol),
                                  make_float2(fmaxf(fabsf(s.x.xy.x), fabsf(xs.xy.x)),
                                              fmaxf(fabsf(s.x.xy.y), fabsf(xs.xy.y))),
                                  bcast(P.atol));
    const float2 scv = __ffma2_rn(bcast(P.rtol),
                                  make_float2(fmaxf(fabsf(s.v.xy.x), fabsf(vn.xy.x)),
                                              fmaxf(fabsf(s.v.xy.y), fabsf(vn.xy.y))),
                                  bcast(P.atol));
    const float2 rx = __fmul2_rn(ex.xy, make_float2(rcp_approx(scx.x), rcp_approx(scx.y)));
    const float2 rv = __fmul2_rn(ev.xy, make_float2(rcp_approx(scv.x), rcp_approx(scv.y)));
    const float2 e2 = __ffma2_rn(rv, rv, __fmul2_rn(rx, rx));
    const float rxz = ex.z * rcp_approx(fmaf(P.rtol, fmaxf(fabsf(s.x.z), fabsf(xs.z)), P.atol));
    const float rvz = ev.z * rcp_approx(fmaf(P.rtol, fmaxf(fabsf(s.v.z), fabsf(vn.z)), P.atol));
    const float errp = fmaf(rvz, rvz, fmaf(rxz, rxz, e2.x + e2.y));
    const float err_sq = gsum<N>(errp, base);
    const Acc pe_new = gsum<N>(pe_half, base);
    int fin_st = -1;
    if (active) {
      // RMS norm squared: en <= 1 exactly when en^2 <= 1, and the controller's
      // en^-1/5 is (en^2)^-1/10, so no square root is taken.
      const float en2 = err_sq * (1.0f / static_cast<float>(6 * N));
      if (en2 <= 1.0f) {
        s.x = xs;
        s.v = vn;
        s.k[0] = a;
        if (L::kKahan) {
          s.cx = cxn;
          s.cv = cvn;
        }
        float factor = (en2 == 0.0f) ? kMaxFactor : fminf(kMaxFactor, kSafety * __powf(en2, 0.5f * kExponent));
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
        const float factor = fmaxf(kMinFactor, kSafety * __powf(en2, 0.5f * kExponent));
        s.h = hh * factor;
        s.rej_once = true;
        s.rejects += 1u;
        s.rej_in_step += 1u;
        if (s.rej_in_step > static_cast<uint32_t>(kMaxRejections)) fin_st = CE_SIM_REJECT_LIMIT;
      }
      if (fin_st >= 0) {
        active = false;
        pending = true;
        s.rej_in_step = static_cast<uint32_t>(fin_st);
        s.pe_stop = pe_new;
      }
    }
  }
}

// Persistent lane-per-atom kernel for one fixed molecule. Block = 32 * W
// threads; no shared memory.
template <int N, int MODE>
__global__ void __launch_bounds__(kAtomMaxBlock) rk45_atom_kernel(const RunParams P, const FixedMol M) {
  const MixedIn none{};
  atom_loop<N, MODE, false, false>(P, M, none, P.cursor, P.S, nullptr, P.refill_threshold);
}

// One size bucket of the one-launch mixed kernel, kept out of line so each
// size gets its own register allocation (inlined into one function, the nine
// loops together needed ~230 registers; apart, the largest needs 128).
template <int N, int MODE>
__device__ __noinline__ void mixed_bucket(const RunParams& P, int refill, const MixedIn X, unsigned long long* cur,
                                          unsigned long long cnt, const uint32_t* perm) {
  const FixedMol none{};
  atom_loop<N, MODE, true, false>(P, none, X, cur, cnt, perm, refill);
}

// Mixed molecules in one persistent launch: every warp walks the size buckets
// from 10 atoms down to 2 (the longest simulations first, and all warps on the
// same N at nearly the same time, so one N's code is hot in the instruction
// cache), serving each bucket from its own queue until it is empty. Four
// blocks per SM are asked for: left free, the nine out-of-line bucket loops
// take 166 registers and only three blocks fit.
template <int MODE>
__global__ void __launch_bounds__(kAtomMaxBlock, 4)
    rk45_mixed_kernel(const __grid_constant__ RunParams P, const MixedIn X, const Buckets B) {
#pragma unroll 1
  for (int n = CE_MAX_ATOMS; n >= 2; --n) {
    const unsigned long long cnt = B.cnt[n];
    if (cnt == 0ull) continue;
    const uint32_t* perm = B.perm + B.off[n];
    unsigned long long* cur = B.cursor + n;
    // the parameters by reference (no per-bucket copy of the kernel arguments)
    const int refill = P.refill_threshold == 0 ? default_refill(n, n) : P.refill_threshold;
    switch (n) {
      case 10: mixed_bucket<10, MODE>(P, refill, X, cur, cnt, perm); break;
      case 9: mixed_bucket<9, MODE>(P, refill, X, cur, cnt, perm); break;
      case 8: mixed_bucket<8, MODE>(P, refill, X, cur, cnt, perm); break;
      case 7: mixed_bucket<7, MODE>(P, refill, X, cur, cnt, perm); break;
      case 6: mixed_bucket<6, MODE>(P, refill, X, cur, cnt, perm); break;
      case 5: mixed_bucket<5, MODE>(P, refill, X, cur, cnt, perm); break;
      case 4: mixed_bucket<4, MODE>(P, refill, X, cur, cnt, perm); break;
      case 3: mixed_bucket<3, MODE>(P, refill, X, cur, cnt, perm); break;
      default: mixed_bucket<2, MODE>(P, refill, X, cur, cnt, perm); break;
    }
  }
}

// One size bucket of a mixed batch (the per-size launch schedule); the only
// kernel that saves and resumes integrator state (RunParams save_* / res_*).
template <int N, int MODE>
__global__ void __launch_bounds__(kAtomMaxBlock) rk45_bucket_kernel(const RunParams P, const MixedIn X, const Buckets B) {
  const FixedMol none{};
  atom_loop<N, MODE, true, true>(P, none, X, B.cursor + N, B.cnt[N], B.perm + B.off[N], P.refill_threshold);
}

using AtomKernelFn = void (*)(RunParams, FixedMol);
AtomKernelFn atom_kernel_m0(int n);
AtomKernelFn atom_kernel_m1(int n);
AtomKernelFn atom_kernel_m2(int n);
AtomKernelFn atom_kernel_m3(int n);

using MixedKernelFn = void (*)(RunParams, MixedIn, Buckets);
// mixed_kernel_m*(0) = the one-launch kernel; mixed_kernel_m*(n), n in 2..10 =
// the single-bucket kernel for n atoms.
MixedKernelFn mixed_kernel_m0(int n);
MixedKernelFn mixed_kernel_m1(int n);
MixedKernelFn mixed_kernel_m2(int n);
MixedKernelFn mixed_kernel_m3(int n);

}  // namespace ce
