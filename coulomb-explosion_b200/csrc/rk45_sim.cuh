// rk45_sim.cuh -- one Coulomb explosion per thread (thread-per-sim layout).
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
//
// Compact attempt loop. The six stage evaluations run in one rolled loop with a
// single inlined force evaluation, so the loop body (a few thousand bytes of
// code for CH4) stays resident in the instruction cache; a fully unrolled
// attempt (six inlined force evaluations) was bound by instruction fetch. The
// loop's stage index is warp-uniform (every thread of a warp runs the same
// stage), so the Butcher coefficients are constant-bank loads at a uniform
// index; stage 7 (x_new, with the potential for the stop test) is peeled out of
// the loop. Stage accelerations live in shared memory, one private
// 16-byte-chunked slot per thread and stage laid out [stage][chunk][thread], so
// a warp's 16-byte accesses touch consecutive addresses (no bank conflicts):
// slots 0..4 hold k2..k6, and k1 and k7 alternate between slots 5 and 6, so the
// FSAL hand-over k1 <- k7 of an accepted step is a slot swap, not a copy. Only x
// and v stay in registers (with k1 there too, CH4 needed more than 128
// registers and spilled).
//
// In-register order of a 3N-vector: the N (x, y) pairs first, then the N z
// components, padded with zeros to whole 16-byte chunks. Every x/y update of the
// pair force and every stage combination then runs on packed FP32x2
// instructions (FFMA2 / FMUL2 / FADD2, per-element IEEE rounding, so results
// equal the scalar formulation).
//
// Two-thread layout (T = 2, rk45_pair_kernel): for 7..10 atoms a whole sim per
// thread needs more registers and stage slots than leave room for enough warps,
// and one lane per atom spends a third of its issue slots on exchange shuffles
// (the SM's shuffle rate bounds it). Two adjacent lanes then share one sim:
// lane h of the pair owns atoms h A .. h A + A - 1 (A = ceil(N / 2)) with the
// same register / stage-slot code as a thread-per-sim run of A atoms, and per
// force evaluation the two lanes swap positions and cross-pair reactions with
// 6A shuffles (pair_forces). Sums over the sim (error norm, potential, kinetic
// energy, initial-step norms) add the partner's part once; IEEE addition is
// commutative, so both lanes hold the identical value and take identical
// decisions. With N odd the second lane's last slot is a phantom atom (charge
// 0, parked 1e15 bohr away): its pair terms are exactly 0, it never moves, and
// it is left out of every norm, sum and output.
#pragma once

#include <cstdint>
#include <type_traits>

#include <cuda_runtime.h>

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
  // Integrator state (lane-per-atom kernels). save_*: written when a sim
  // finishes, the state it stopped in (save_h = 0 unless it finished
  // CE_SIM_OK). res_*: when res_h is non-null, a sim whose res_h > 0 starts
  // from that state (positions res_pos) instead of from rest, and continues
  // exactly as the run that saved it would have; the others start from rest.
  float* save_pos;     // [S][stride][3]
  float* save_vel;     // [S][stride][3] v (not m v)
  float* save_h;       // [S] next step size
  double* save_t;      // [S]
  uint32_t* save_steps;
  uint32_t* save_rejects;
  double* save_e0;
  float* save_comp;    // [S][stride][6] Kahan compensation of x (0..2) and v (3..5)
  const float* res_pos;
  const float* res_vel;
  const float* res_h;
  const double* res_t;
  const uint32_t* res_steps;
  const uint32_t* res_rejects;
  const double* res_e0;
  const float* res_comp;
  // Streamed host-buffer run (ce_run, the *_io kernels): positions arrive in
  // chunks of 2^io_shift sims, io_ready[j] != 0 once chunk j is in device memory
  // (written by a copy after the chunk's own copy). Every finished sim is
  // counted in io_done[j] (one count per thread of the sim); the count that
  // completes chunk j raises io_host_done[j] in mapped host memory, and the host
  // then copies that chunk's results out. io_abort (mapped host memory) != 0 ends
  // every input wait at once; a wait that ends without its input sets io_error
  // (mapped host memory) and its sims finish as CE_SIM_BAD_INPUT.
  const unsigned* io_ready;
  unsigned long long* io_done;
  unsigned* io_host_done;
  const unsigned* io_abort;
  unsigned* io_error;
  unsigned io_shift;  // chunks of 2^io_shift sims
};

constexpr int kMixedStride = CE_MAX_ATOMS;  // atoms per sim row in the mixed layout

// Per-sim molecule arrays of the mixed layout (rows of kMixedStride atoms).
struct MixedIn {
  const uint8_t* n_per;   // [S] atoms per sim
  const double* mass;     // [S][10] electron masses
  const double* charge;   // [S][10]
  double coulomb_k;
};

// Size buckets produced by the device counting sort (mixed.cu): sims of size n
// are perm[off[n] .. off[n] + cnt[n]); cursor[n] is that bucket's work queue.
struct Buckets {
  const uint32_t* perm;
  const unsigned long long* off;  // [11]
  const unsigned long long* cnt;  // [11]
  unsigned long long* cursor;     // [11]
};

// Variants of the thread-per-sim / two-thread loop (template flags):
//   kLoopIO     streamed host-buffer I/O (RunParams io_*)
//   kLoopMixed  a mixed batch: rows of kMixedStride atoms, each sim's masses and
//               charges from its row (two threads per sim only)
//   kLoopState  saved / resumed integrator state (RunParams save_* / res_*)
constexpr int kLoopIO = 1, kLoopMixed = 2, kLoopState = 4;


// Packed-FP32x2 helpers (sm_100: FFMA2 / FMUL2 / FADD2; every element rounds
// exactly like the scalar instruction) and the approximate MUFU forms.
__device__ __forceinline__ float2 bcast(float s) { return make_float2(s, s); }

// Packed operations on float pair p of a register vector with NF real floats
// (p a compile-time index after unrolling): both halves in one FFMA2 / FMUL2 /
// FADD2 while both are real; when NF is odd the last real float alone in a
// scalar instruction, its padding half left as it is; a pair of padding alone is
// left untouched. A padding half would otherwise take an FMA-pipe slot of its own.
template <int NF>
__device__ __forceinline__ float2 pfma(int p, float2 a, float2 b, float2 c) {
  if (2 * p + 1 < NF) return __ffma2_rn(a, b, c);
  if (2 * p < NF) return make_float2(fmaf(a.x, b.x, c.x), c.y);
  return c;
}
template <int NF>
__device__ __forceinline__ float2 pmul(int p, float2 a, float2 b) {
  if (2 * p + 1 < NF) return __fmul2_rn(a, b);
  if (2 * p < NF) return make_float2(a.x * b.x, 0.0f);
  return make_float2(0.0f, 0.0f);
}
template <int NF>
__device__ __forceinline__ float2 padd(int p, float2 a, float2 b) {
  if (2 * p + 1 < NF) return __fadd2_rn(a, b);
  if (2 * p < NF) return make_float2(a.x + b.x, a.y);
  return a;
}

// Approximate reciprocal and square root (PTX rcp.approx / sqrt.approx, flush
// to zero): for the error-norm scales and the initial-step heuristic, where a
// relative error of a few 1e-7 changes no decision the integrator relies on.
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Register and shared-memory shape of one simulation in the thread-per-sim layout.
template <int N>
struct ThreadShape {
  static constexpr int NF = 3 * N;         // floats of a 3N-vector
  static constexpr int NC = (NF + 3) / 4;  // 16-byte chunks per stage slot
  static constexpr int NP = 2 * NC;        // float2 register pairs (zero-padded)
  static constexpr int kSlots = 7;         // k2..k6, and k1 / k7 alternating between two slots
  // Blocks of kThreadMaxBlock threads per SM the register allocator aims for:
  // 128 registers a thread for CH4-sized molecules, more for larger N (whose
  // shared-memory slots allow fewer blocks anyway).
  static constexpr int kMinBlocks = N <= 5 ? 4 : (N <= 7 ? 3 : 2);
};

// One thread's share of a simulation: T threads per sim (1, or 2 for the
// two-thread layout), A atoms a thread; ThreadShape<A> sizes its registers and
// stage slots. With T = 2 and N odd the second thread's last slot is a phantom.
template <int N, int T>
struct SimShape {
  static constexpr int A = (N + T - 1) / T;
  static constexpr int NF = 3 * A;
  static constexpr int NC = (NF + 3) / 4;
  static constexpr int NP = 2 * NC;
  static constexpr bool kPhantom = T * A != N;
};

// Stage slots per thread: k2..k6 and k1 / k7 (7); with Kahan compensation also
// cx and cv, each alternating between two slots like k1 / k7 (11).
__host__ __device__ constexpr int thread_slots(int mode) { return (mode & CE_PREC_KAHAN) ? 11 : 7; }
// Blocks per SM the register allocator aims for; with the Kahan slots the
// shared memory allows fewer blocks, so more registers a thread.
template <int N, int MODE>
__host__ __device__ constexpr int thread_min_blocks() {
  return N >= 8 ? 4 : ((MODE & CE_PREC_KAHAN) ? (N <= 4 ? 3 : 2) : ThreadShape<N>::kMinBlocks);
}

constexpr int kThreadMaxBlock = 128;
// Threads per block of the thread-per-sim kernel: 128, and 64 from 8 atoms up,
// where a 128-thread block's stage slots would leave room for one block per SM.
__host__ __device__ constexpr int thread_block(int n) { return n >= 8 ? 64 : kThreadMaxBlock; }

// Dynamic shared memory of one thread-per-sim block: thread_slots(mode) stage
// slots of NC 16-byte chunks for each of its threads (n = atoms a thread).
__host__ __device__ constexpr size_t thread_smem_bytes(int n, int block, int mode) {
  return static_cast<size_t>(thread_slots(mode)) * static_cast<size_t>((3 * n + 3) / 4) * 16u *
         static_cast<size_t>(block);
}

// Two-thread layout: 128-thread blocks (64 sims), at most 5 atoms a thread.
constexpr int kPairBlock = 128;
__host__ __device__ constexpr int pair_atoms(int n) { return (n + 1) / 2; }
__host__ __device__ constexpr size_t pair_smem_bytes(int n, int mode) {
  return thread_smem_bytes(pair_atoms(n), kPairBlock, mode);
}
// Blocks per SM the two-thread kernel's register allocator aims for: five
// atoms a thread (9 and 10 atoms) take 168 registers at 3 blocks (C2H6-like,
// 1e6 sims at the tight point: 7.49e7 explosions/s against 6.76e7 at 128
// registers with spills); with the Kahan slots shared memory allows 2 blocks.
template <int N, int MODE>
__host__ __device__ constexpr int pair_min_blocks() {
  return (SimShape<N, 2>::A >= 5 && (MODE & CE_PREC_KAHAN) == 0) ? 3 : thread_min_blocks<SimShape<N, 2>::A, MODE>();
}
// Threads per block of the T-threads-per-sim kernels (fixed at compile time:
// the stage-slot offsets are immediates).
template <int N, int T>
__host__ __device__ constexpr int sim_block() {
  return T == 2 ? kPairBlock : thread_block(N);
}

// Flat float f of a register 3N-vector (x_i at 2i, y_i at 2i + 1, z_i at 2N + i);
// f is a compile-time index after unrolling (values, never addresses, so the
// arrays stay in registers).
template <int NP>
__device__ __forceinline__ void fl_set(float2 (&r)[NP], int f, float val) {
  const float2 t = r[f >> 1];
  r[f >> 1] = (f & 1) ? make_float2(t.x, val) : make_float2(val, t.y);
}
template <int NP>
__device__ __forceinline__ float flc(const float2 (&r)[NP], int f) {
  const float2 t = r[f >> 1];  // select between values, not addresses
  return (f & 1) ? t.y : t.x;
}
__device__ __forceinline__ constexpr int flat_of(int n, int i, int c) { return c < 2 ? 2 * i + c : 2 * n + i; }

// a_i = (1/m_i) sum_j k q_i q_j r_ij / |r_ij|^3 with Newton's third law, and
// (if want_pe) pe += sum_{i<j} k q_i q_j / |r_ij|. Pairs in i < j order, each
// acceleration accumulated from zero in that order (the order of
// src/system.cpp:5-25); the x/y halves of every update are one FFMA2.
template <int N, typename TPE>
__device__ __forceinline__ void thread_forces(const float2 (&x)[ThreadShape<N>::NP],
                                              float2 (&a)[ThreadShape<N>::NP], const FixedMol& M,
                                              bool want_pe, TPE& pe) {
  constexpr int NP = ThreadShape<N>::NP;
  float2 axy[N];
  float az[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    axy[i] = make_float2(0.0f, 0.0f);
    az[i] = 0.0f;
  }
#pragma unroll
  for (int i = 0; i < N; ++i) {
#pragma unroll
    for (int j = 0; j < N; ++j) {
      if (j <= i) continue;  // constant trip count: the unrolled pair loop keeps every array in registers
      const float2 rxy = __ffma2_rn(bcast(-1.0f), x[j], x[i]);
      const float rz = flc<NP>(x, 2 * N + i) - flc<NP>(x, 2 * N + j);
      const float d2 = fmaf(rxy.x, rxy.x, fmaf(rxy.y, rxy.y, rz * rz));
      const float rinv = rsqrtf(d2);
      const float u = M.pc[i * N + j] * rinv;  // pair potential k q_i q_j / r
      if (want_pe) pe += static_cast<TPE>(u);
      const float sc = u * (rinv * rinv);      // k q_i q_j / r^3
      axy[i] = __ffma2_rn(rxy, bcast(sc), axy[i]);
      az[i] = fmaf(rz, sc, az[i]);
      axy[j] = __ffma2_rn(rxy, bcast(-sc), axy[j]);
      az[j] = fmaf(-rz, sc, az[j]);
    }
  }
#pragma unroll
  for (int i = 0; i < N; ++i) {
    // scalar products with the constant-bank 1/m_i (a packed product would first
    // copy it into a register pair)
    a[i] = make_float2(axy[i].x * M.inv_m[i], axy[i].y * M.inv_m[i]);
    fl_set<NP>(a, 2 * N + i, az[i] * M.inv_m[i]);
  }
#pragma unroll
  for (int f = 3 * N; f < 2 * NP; ++f) fl_set<NP>(a, f, 0.0f);
}

// Cross pairs of the two-thread layout. Thread h owns atoms h A + a (slots
// a = 0..A-1) and sees its partner's atoms in the same slots b. It evaluates
// the cross pair (own a, partner b) for b - a = d (mod A) with d = 0 (both
// threads evaluate these; each keeps its own side and half the potential),
// 0 < 2d < A, and 2d = A when a < A/2. The partner evaluates the mirror
// offsets -d, so every other cross pair is evaluated by exactly one thread,
// which hands the reaction -f to the other (Newton's third law).
__host__ __device__ constexpr bool pair_cross(int A, int b, int d) {
  return d == 0 || 2 * d < A || (2 * d == A && (b - d + A) % A < A / 2);
}
template <int A>
__host__ __device__ constexpr int pair_cross_count() {
  int c = 0;
  for (int b = 0; b < A; ++b)
    for (int d = 0; d < A; ++d)
      if (pair_cross(A, b, d)) ++c;
  return c;
}

// One thread's constants in the two-thread layout, in registers (the two
// threads of a pair own different atoms, so a constant-bank operand at a
// compile-time index cannot serve both): k q_i q_j of its own pairs (i < j
// order) and of the cross pairs it evaluates (pair_forces' loop order), 1/m of
// its atoms. Phantom entries are 0 (1 for 1/m).
struct NoConsts {};
template <int N>
struct PairConsts {
  static constexpr int A = SimShape<N, 2>::A;
  static constexpr int NI = A * (A - 1) / 2;
  static constexpr int NX = pair_cross_count<A>();
  float pcI[NI > 0 ? NI : 1];
  float pcX[NX];
  float inv_m[A];
  int half;        // 0 or 1: which half of the sim's atoms this thread owns
  unsigned pmask;  // this thread's lane and its partner's
};
template <int N, int T>
using SimConsts = typename std::conditional<T == 2, PairConsts<N>, NoConsts>::type;

template <int N>
__device__ __forceinline__ void load_pair_consts(PairConsts<N>& C, const FixedMol& M, unsigned lane) {
  constexpr int A = PairConsts<N>::A;
  C.half = static_cast<int>(lane & 1u);
  C.pmask = 3u << (lane & 30u);
  const int o = C.half * A, po = (1 - C.half) * A;
  int k = 0;
#pragma unroll
  for (int i = 0; i < A; ++i)
#pragma unroll
    for (int j = 0; j < A; ++j) {
      if (j <= i) continue;
      C.pcI[k++] = (o + j < N) ? M.pc[(o + i) * N + o + j] : 0.0f;
    }
  k = 0;
#pragma unroll
  for (int b = 0; b < A; ++b)
#pragma unroll
    for (int d = 0; d < A; ++d) {
      if (!pair_cross(A, b, d)) continue;
      const int i = (b - d + A) % A;
      C.pcX[k++] = (o + i < N && po + b < N) ? M.pc[(o + i) * N + po + b] : 0.0f;
    }
#pragma unroll
  for (int a = 0; a < A; ++a) C.inv_m[a] = (o + a < N) ? M.inv_m[o + a] : 1.0f;
}

// The same constants for mixed-batch sim `sim`, from its row: k q_i q_j formed
// in double and narrowed, 1/m narrowed, as ce_set_molecule forms them for the
// fixed path. C.half and C.pmask are already set.
template <int N>
__device__ __forceinline__ void load_pair_consts_mixed(PairConsts<N>& C, const MixedIn& X, unsigned long long sim) {
  constexpr int A = PairConsts<N>::A;
  const int o = C.half * A, po = (1 - C.half) * A;
  const double* q = X.charge + sim * kMixedStride;
  const double* m = X.mass + sim * kMixedStride;
  double qo[A], qp[A];
#pragma unroll
  for (int a = 0; a < A; ++a) {
    qo[a] = (o + a < N) ? __ldg(q + o + a) : 0.0;
    qp[a] = (po + a < N) ? __ldg(q + po + a) : 0.0;
    C.inv_m[a] = (o + a < N) ? static_cast<float>(1.0 / __ldg(m + o + a)) : 1.0f;
  }
  int k = 0;
#pragma unroll
  for (int i = 0; i < A; ++i)
#pragma unroll
    for (int j = 0; j < A; ++j) {
      if (j <= i) continue;
      C.pcI[k++] = static_cast<float>(X.coulomb_k * qo[i] * qo[j]);
    }
  k = 0;
#pragma unroll
  for (int b = 0; b < A; ++b)
#pragma unroll
    for (int d = 0; d < A; ++d) {
      if (!pair_cross(A, b, d)) continue;
      C.pcX[k++] = static_cast<float>(X.coulomb_k * qo[(b - d + A) % A] * qp[b]);
    }
}

// m_i (double) of atom i of sim `sim`.
template <bool MIXED>
__device__ __forceinline__ double sim_mass(const FixedMol& M, const MixedIn& X, unsigned long long sim, int i) {
  if constexpr (MIXED)
    return __ldg(X.mass + sim * kMixedStride + i);
  else
    return M.mass[i];
}

// a for this thread's A atoms in the two-thread layout: its own pairs as in
// thread_forces, then the cross pairs partner slot by partner slot: the
// partner's position of slot b arrives by three shuffles, the pairs
// (b - d, b) of pair_cross are evaluated, and the reactions this thread
// collected for the partner's atom b are swapped for the ones the partner
// collected for this thread's atom b (three more shuffles). pe gets this
// thread's share of the potential (its own pairs, its cross pairs, half of
// each d = 0 pair); the two shares add up to PE.
template <int N, typename TPE>
__device__ __forceinline__ void pair_forces(const float2 (&x)[SimShape<N, 2>::NP], float2 (&a)[SimShape<N, 2>::NP],
                                            const PairConsts<N>& C, bool want_pe, TPE& pe) {
  constexpr int A = SimShape<N, 2>::A;
  constexpr int NP = SimShape<N, 2>::NP;
  float2 axy[A];
  float az[A];
#pragma unroll
  for (int i = 0; i < A; ++i) {
    axy[i] = make_float2(0.0f, 0.0f);
    az[i] = 0.0f;
  }
  int k = 0;
#pragma unroll
  for (int i = 0; i < A; ++i) {
#pragma unroll
    for (int j = 0; j < A; ++j) {
      if (j <= i) continue;
      const float2 rxy = __ffma2_rn(bcast(-1.0f), x[j], x[i]);
      const float rz = flc<NP>(x, 2 * A + i) - flc<NP>(x, 2 * A + j);
      const float d2 = fmaf(rxy.x, rxy.x, fmaf(rxy.y, rxy.y, rz * rz));
      const float rinv = rsqrtf(d2);
      const float u = C.pcI[k++] * rinv;
      if (want_pe) pe += static_cast<TPE>(u);
      const float sc = u * (rinv * rinv);
      axy[i] = __ffma2_rn(rxy, bcast(sc), axy[i]);
      az[i] = fmaf(rz, sc, az[i]);
      axy[j] = __ffma2_rn(rxy, bcast(-sc), axy[j]);
      az[j] = fmaf(-rz, sc, az[j]);
    }
  }
  k = 0;
#pragma unroll
  for (int b = 0; b < A; ++b) {
    const float2 pxy = make_float2(__shfl_xor_sync(C.pmask, x[b].x, 1), __shfl_xor_sync(C.pmask, x[b].y, 1));
    const float pz = __shfl_xor_sync(C.pmask, flc<NP>(x, 2 * A + b), 1);
    float2 rbxy = make_float2(0.0f, 0.0f);  // reaction on the partner's atom b
    float rbz = 0.0f;
#pragma unroll
    for (int d = 0; d < A; ++d) {
      if (!pair_cross(A, b, d)) continue;
      const int i = (b - d + A) % A;
      const float2 rxy = __ffma2_rn(bcast(-1.0f), pxy, x[i]);
      const float rz = flc<NP>(x, 2 * A + i) - pz;
      const float d2 = fmaf(rxy.x, rxy.x, fmaf(rxy.y, rxy.y, rz * rz));
      const float rinv = rsqrtf(d2);
      const float u = C.pcX[k++] * rinv;
      if (want_pe) pe += static_cast<TPE>(d == 0 ? 0.5f * u : u);
      const float sc = u * (rinv * rinv);
      axy[i] = __ffma2_rn(rxy, bcast(sc), axy[i]);
      az[i] = fmaf(rz, sc, az[i]);
      if (d != 0) {
        rbxy = __ffma2_rn(rxy, bcast(-sc), rbxy);
        rbz = fmaf(-rz, sc, rbz);
      }
    }
    const float2 gxy = make_float2(__shfl_xor_sync(C.pmask, rbxy.x, 1), __shfl_xor_sync(C.pmask, rbxy.y, 1));
    axy[b] = __fadd2_rn(axy[b], gxy);
    az[b] += __shfl_xor_sync(C.pmask, rbz, 1);
  }
#pragma unroll
  for (int i = 0; i < A; ++i) {
    a[i] = make_float2(axy[i].x * C.inv_m[i], axy[i].y * C.inv_m[i]);
    fl_set<NP>(a, 2 * A + i, az[i] * C.inv_m[i]);
  }
#pragma unroll
  for (int f = 3 * A; f < 2 * NP; ++f) fl_set<NP>(a, f, 0.0f);
}

// The force evaluation of a T-threads-per-sim run.
template <int N, int T, typename TPE>
__device__ __forceinline__ void sim_forces(const float2 (&x)[SimShape<N, T>::NP], float2 (&a)[SimShape<N, T>::NP],
                                           const FixedMol& M, const SimConsts<N, T>& C, bool want_pe, TPE& pe) {
  if constexpr (T == 2)
    pair_forces<N, TPE>(x, a, C, want_pe, pe);
  else
    thread_forces<N, TPE>(x, a, M, want_pe, pe);
}

// Sum of a per-thread part over the T threads of a sim (v + partner's v: the
// same bits in both threads).
template <int N, int T, typename V>
__device__ __forceinline__ V sim_sum(V v, const SimConsts<N, T>& C) {
  if constexpr (T == 2)
    return v + __shfl_xor_sync(C.pmask, v, 1);
  else
    return v;
}

// Whether flat float f of thread `half`'s register vector belongs to a real
// atom (false only for the phantom slot).
template <int N, int T>
__device__ __forceinline__ bool sim_real(int f, int half) {
  constexpr int A = SimShape<N, T>::A;
  if constexpr (!SimShape<N, T>::kPhantom) return true;
  const int atom = f < 2 * A ? (f >> 1) : f - 2 * A;
  return half == 0 || atom != A - 1;
}

template <int N, int MODE, int T = 1>
struct ThreadSim {
  static constexpr bool kKahan = (MODE & CE_PREC_KAHAN) != 0;
  static constexpr bool kF64 = (MODE & CE_PREC_FP64) != 0;
  static constexpr int NP = SimShape<N, T>::NP;

  using Acc = typename std::conditional<kF64, double, float>::type;

  float2 x[NP];
  float2 v[NP];
  int k1s;        // stage slot holding k1 = a(x) (FSAL): 5 or 6; k7 goes to the other
  int cxs, cvs;   // stage slots holding the Kahan compensation of x (7 or 8) and v (9 or 10)
  float h;
  Acc t;
  Acc e0;
  Acc pe_stop;
  uint32_t steps, rejects, rej_in_step;
  bool rej_once;
  unsigned long long sim;
};

// Stores the first K floats of v (K compile-time) with float2 stores: an 8-byte
// aligned start writes pairs (and a trailing single when K is odd), a start 4
// bytes past alignment writes one single first.
template <int K, int L>
__device__ __forceinline__ void store_record(float* dst, const float (&v)[L]) {
  static_assert(K <= L, "store_record: record longer than its source");
  if ((reinterpret_cast<uintptr_t>(dst) & 7u) == 0u) {
#pragma unroll
    for (int f = 0; f + 1 < K; f += 2) *reinterpret_cast<float2*>(dst + f) = make_float2(v[f], v[f + 1]);
    if (K & 1) dst[K - 1] = v[K - 1];
  } else {
    dst[0] = v[0];
#pragma unroll
    for (int f = 1; f + 1 < K; f += 2) *reinterpret_cast<float2*>(dst + f) = make_float2(v[f], v[f + 1]);
    if (!(K & 1)) dst[K - 1] = v[K - 1];
  }
}

// Flat float f of the 16-byte-chunked stage slot `slot` of this thread (B
// threads per block).
template <int NC, int B>
__device__ __forceinline__ float slot_float(const float4* ks, int slot, int f) {
  return reinterpret_cast<const float*>(ks + (slot * NC + (f >> 2)) * B)[f & 3];
}

// FP64 finalize: KE, s = sqrt(E0/KE), p_i = (m_i s) v_i, KER = s^2 KE; then the
// per-sim output record (rows of N atoms, or kMixedStride in a mixed batch)
// and, with kLoopState, the integrator state the sim stopped in (RunParams
// save_*). A converged sim with non-finite momenta is CE_SIM_NONFINITE. In the
// two-thread layout each thread writes its own atoms' rows and thread 0 the
// per-sim scalars.
template <int N, int MODE, int T, int F>
__device__ __forceinline__ void thread_finalize(const ThreadSim<N, MODE, T>& s, int status, double pe_final,
                                                const RunParams& P, const FixedMol& M, const MixedIn& X,
                                                const SimConsts<N, T>& C, const float4* ks) {
  constexpr int A = SimShape<N, T>::A;
  constexpr int NP = SimShape<N, T>::NP;
  constexpr bool MIXED = (F & kLoopMixed) != 0;
  constexpr int STRIDE = MIXED ? kMixedStride : N;
  int half = 0;
  if constexpr (T == 2) half = C.half;
  const int o = half * A;  // first atom of this thread
  double ke = 0.0;
  bool finite = true;
#pragma unroll
  for (int i = 0; i < A; ++i) {
    if (!sim_real<N, T>(2 * i, half)) continue;
    const double vx = s.v[i].x, vy = s.v[i].y, vz = flc<NP>(s.v, 2 * A + i);
    ke += 0.5 * sim_mass<MIXED>(M, X, s.sim, o + i) * (vx * vx + vy * vy + vz * vz);
    finite = finite && isfinite(vx) && isfinite(vy) && isfinite(vz);
  }
  if constexpr (T == 2) {
    ke = sim_sum<N, T>(ke, C);
    finite = (__shfl_xor_sync(C.pmask, finite ? 1 : 0, 1) != 0) && finite;
  }
  if (status == CE_SIM_OK && !finite) status = CE_SIM_NONFINITE;
  const double e0d = static_cast<double>(s.e0);
  const double sc =
      (P.redistribute && ke > 0.0) ? (e0d > 0.0 ? e0d * rsqrt(e0d * ke) : sqrt(e0d / ke)) : 1.0;
  // The momenta, written as one contiguous record with 8-byte stores (a record
  // starts 8-byte aligned or 4 bytes past it, depending on the sim).
  float pm[3 * A];
#pragma unroll
  for (int i = 0; i < A; ++i) {
    const double mm = (sim_real<N, T>(2 * i, half) ? sim_mass<MIXED>(M, X, s.sim, o + i) : 0.0) * sc;
    pm[i * 3 + 0] = static_cast<float>(mm * static_cast<double>(s.v[i].x));
    pm[i * 3 + 1] = static_cast<float>(mm * static_cast<double>(s.v[i].y));
    pm[i * 3 + 2] = static_cast<float>(mm * static_cast<double>(flc<NP>(s.v, 2 * A + i)));
  }
  const unsigned long long row = s.sim * (3ull * STRIDE) + 3 * o;  // this thread's first float of the sim's rows
  if (SimShape<N, T>::kPhantom && half == 1)
    store_record<3 * (A - 1)>(P.momenta + row, pm);
  else
    store_record<3 * A>(P.momenta + row, pm);
  if (half == 0) {
    if (P.ker) P.ker[s.sim] = (sc * sc) * ke;
    if (P.steps) P.steps[s.sim] = s.steps;
    if (P.status) P.status[s.sim] = static_cast<uint8_t>(status);
    if (P.rejects) P.rejects[s.sim] = s.rejects;
    if (P.t_final) P.t_final[s.sim] = static_cast<double>(s.t);
    if (P.pe_final) P.pe_final[s.sim] = pe_final;
    if (P.ke_before) P.ke_before[s.sim] = ke;
    if (P.e0) P.e0[s.sim] = e0d;
  }
  if (P.positions) {
#pragma unroll
    for (int i = 0; i < A; ++i) {
      if (!sim_real<N, T>(2 * i, half)) continue;
      P.positions[row + i * 3 + 0] = s.x[i].x;
      P.positions[row + i * 3 + 1] = s.x[i].y;
      P.positions[row + i * 3 + 2] = flc<NP>(s.x, 2 * A + i);
    }
  }
  if constexpr ((F & kLoopState) != 0) {
    if (P.save_h) {  // the integrator state this sim stopped in (a resumable run's input)
      constexpr int NC = SimShape<N, T>::NC;
      constexpr int B = sim_block<N, T>();
#pragma unroll
      for (int i = 0; i < A; ++i) {
        if (!sim_real<N, T>(2 * i, half)) continue;
        P.save_pos[row + i * 3 + 0] = s.x[i].x;
        P.save_pos[row + i * 3 + 1] = s.x[i].y;
        P.save_pos[row + i * 3 + 2] = flc<NP>(s.x, 2 * A + i);
        P.save_vel[row + i * 3 + 0] = s.v[i].x;
        P.save_vel[row + i * 3 + 1] = s.v[i].y;
        P.save_vel[row + i * 3 + 2] = flc<NP>(s.v, 2 * A + i);
        if (ThreadSim<N, MODE, T>::kKahan && P.save_comp) {
          float* c = P.save_comp + s.sim * (6ull * STRIDE) + 6 * (o + i);
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const int f = flat_of(A, i, k);
            c[k] = slot_float<NC, B>(ks, s.cxs, f);
            c[3 + k] = slot_float<NC, B>(ks, s.cvs, f);
          }
        }
      }
      if (half == 0) {
        P.save_h[s.sim] = status == CE_SIM_OK ? s.h : 0.0f;
        P.save_t[s.sim] = static_cast<double>(s.t);
        P.save_steps[s.sim] = s.steps;
        P.save_rejects[s.sim] = s.rejects;
        P.save_e0[s.sim] = e0d;
      }
    }
  }
}

// Load sim `sim`, evaluate k1 (into stage slot 5) and PE0 and choose the first step (Hairer's
// heuristic from rest, src/integrators.cpp:197-250 with v0 = 0: every velocity
// term is 0, sv = atol, and the probe accelerations equal k1; its quotients use
// the fast forms, as the initial step is a heuristic). Returns false when the
// sim is already finished (written out). In the two-thread layout both
// threads of the pair run it for their own atoms. In a mixed batch
// (kLoopMixed) the sim's constants come from its row of X (C is reloaded);
// with kLoopState a sim whose res_h > 0 resumes its saved state instead
// (positions, velocities, compensation, step size, clock, counters, E_0): its
// k1 = a(x) is bit for bit the k7 of the accepted step the state follows, and
// the driver's stop test runs again on the current potential
// (src/driver.cpp:19-30), as the uninterrupted run would.
template <int N, int MODE, int T, int F>
__device__ __forceinline__ bool thread_init(ThreadSim<N, MODE, T>& s, unsigned long long sim, const RunParams& P,
                                            const FixedMol& M, const MixedIn& X, SimConsts<N, T>& C, float4* ks,
                                            int B) {
  using S = ThreadSim<N, MODE, T>;
  using Acc = typename S::Acc;
  constexpr int A = SimShape<N, T>::A;
  constexpr int NP = SimShape<N, T>::NP;
  constexpr int NC = SimShape<N, T>::NC;
  constexpr bool IO = (F & kLoopIO) != 0;
  constexpr bool MIXED = (F & kLoopMixed) != 0;
  constexpr bool STATE = (F & kLoopState) != 0;
  constexpr int STRIDE = MIXED ? kMixedStride : N;
  static_assert(!MIXED || T == 2, "mixed batches run the two-thread layout here");
  int half = 0;
  if constexpr (T == 2) half = C.half;
  s.sim = sim;
  bool resumed = false;
  if constexpr (STATE) resumed = P.res_h != nullptr && __ldg(P.res_h + sim) > 0.0f;
  const unsigned long long row = sim * (3ull * STRIDE) + 3 * (half * A);
  const float* src = (resumed ? P.res_pos : P.pos) + row;
#pragma unroll
  for (int p = 0; p < NP; ++p) s.x[p] = s.v[p] = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int i = 0; i < A; ++i) {
    if (!sim_real<N, T>(2 * i, half)) {  // the phantom: zero charge, parked far from every atom
      s.x[i] = make_float2(1e15f, 1e15f);
      fl_set<NP>(s.x, 2 * A + i, 1e15f);
    } else if (IO) {  // written by a copy while the kernel runs: plain (coherent) loads after the
                      // acquire that saw the chunk present, not the read-only path
      s.x[i] = make_float2(src[3 * i], src[3 * i + 1]);
      fl_set<NP>(s.x, 2 * A + i, src[3 * i + 2]);
    } else {
      s.x[i] = make_float2(__ldg(src + 3 * i), __ldg(src + 3 * i + 1));
      fl_set<NP>(s.x, 2 * A + i, __ldg(src + 3 * i + 2));
    }
  }
  if constexpr (STATE) {
    if (resumed) {
#pragma unroll
      for (int i = 0; i < A; ++i) {
        if (!sim_real<N, T>(2 * i, half)) continue;
        const float* vs = P.res_vel + row;
        s.v[i] = make_float2(__ldg(vs + 3 * i), __ldg(vs + 3 * i + 1));
        fl_set<NP>(s.v, 2 * A + i, __ldg(vs + 3 * i + 2));
      }
    }
  }
  if (S::kKahan) {  // compensation terms start at zero (or from the saved state)
    s.cxs = 7;
    s.cvs = 9;
    float2 cx[NP], cv[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) cx[p] = cv[p] = make_float2(0.0f, 0.0f);
    if constexpr (STATE) {
      if (resumed) {
#pragma unroll
        for (int i = 0; i < A; ++i) {
          if (!sim_real<N, T>(2 * i, half)) continue;
          const float* c = P.res_comp + sim * (6ull * STRIDE) + 6 * (half * A + i);
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            fl_set<NP>(cx, flat_of(A, i, k), __ldg(c + k));
            fl_set<NP>(cv, flat_of(A, i, k), __ldg(c + 3 + k));
          }
        }
      }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      ks[(7 * NC + c) * B] = make_float4(cx[2 * c].x, cx[2 * c].y, cx[2 * c + 1].x, cx[2 * c + 1].y);
      ks[(9 * NC + c) * B] = make_float4(cv[2 * c].x, cv[2 * c].y, cv[2 * c + 1].x, cv[2 * c + 1].y);
    }
  }
  if constexpr (MIXED) load_pair_consts_mixed<N>(C, X, sim);
  Acc pe0 = Acc(0);
  float2 k0[NP];
  sim_forces<N, T, Acc>(s.x, k0, M, C, true, pe0);
  pe0 = sim_sum<N, T>(pe0, C);
  s.k1s = 5;
#pragma unroll
  for (int c = 0; c < NC; ++c)
    ks[(5 * NC + c) * B] = make_float4(k0[2 * c].x, k0[2 * c].y, k0[2 * c + 1].x, k0[2 * c + 1].y);
  if constexpr (STATE) {
    if (resumed) {
      s.h = __ldg(P.res_h + sim);
      s.t = static_cast<Acc>(P.res_t[sim]);
      s.steps = P.res_steps[sim];
      s.rejects = P.res_rejects[sim];
      s.rej_in_step = 0u;
      s.rej_once = false;
      s.e0 = static_cast<Acc>(P.res_e0[sim]);
      if (S::kF64)
        s.pe_stop = static_cast<Acc>(P.pe_stop_d * static_cast<double>(s.e0));
      else
        s.pe_stop = static_cast<Acc>(P.pe_stop_f * static_cast<float>(s.e0));
      int fin = -1;
      if (!(pe0 > s.pe_stop)) fin = CE_SIM_OK;
      else if (s.steps >= P.max_steps) fin = CE_SIM_MAX_STEPS;
      if (fin >= 0) {
        thread_finalize<N, MODE, T, F>(s, fin, static_cast<double>(pe0), P, M, X, C, ks);
        return false;
      }
      return true;
    }
  }
  s.t = Acc(0);
  s.steps = s.rejects = s.rej_in_step = 0u;
  s.rej_once = false;
  s.e0 = pe0;  // E_0 = PE_0 + KE_0, KE_0 = 0 (batched_integrator.hpp:137)
  if (S::kF64)
    s.pe_stop = static_cast<Acc>(P.pe_stop_d * static_cast<double>(pe0));
  else
    s.pe_stop = static_cast<Acc>(P.pe_stop_f * static_cast<float>(pe0));
  int fin = -1;
  if (!isfinite(static_cast<double>(pe0))) fin = CE_SIM_NONFINITE;
  else if (!(pe0 > s.pe_stop)) fin = CE_SIM_OK;  // already at or below the stop (driver.cpp:19)
  else if (P.max_steps == 0u) fin = CE_SIM_MAX_STEPS;
  if (fin >= 0) {
    thread_finalize<N, MODE, T, F>(s, fin, static_cast<double>(pe0), P, M, X, C, ks);
    return false;
  }
  float d0_sq = 0.0f, d1_sq = 0.0f;
  const float inv_atol = __frcp_rn(P.atol);
#pragma unroll
  for (int f = 0; f < 3 * A; ++f) {
    const float xf = flc<NP>(s.x, f);
    const float r0 = __fdividef(xf, P.atol + P.rtol * fabsf(xf));
    const float r1 = flc<NP>(k0, f) * inv_atol;
    if (sim_real<N, T>(f, half)) d0_sq += r0 * r0;
    d1_sq += r1 * r1;
  }
  d0_sq = sim_sum<N, T>(d0_sq, C);
  d1_sq = sim_sum<N, T>(d1_sq, C);
  constexpr float inv_denom = 1.0f / static_cast<float>(6 * N);
  const float d0 = sqrt_approx(d0_sq * inv_denom);
  const float d1 = sqrt_approx(d1_sq * inv_denom);
  const float h0 = (static_cast<double>(d0) < 1e-5 || static_cast<double>(d1) < 1e-5) ? 1e-6f
                                                                                         : __fdividef(0.01f * d0, d1);
  float d2_sq = 0.0f;
#pragma unroll
  for (int f = 0; f < 3 * A; ++f) {
    const float xf = flc<NP>(s.x, f);
    const float r = __fdividef(flc<NP>(k0, f) * h0, P.atol + P.rtol * fabsf(xf));
    d2_sq += r * r;
  }
  d2_sq = sim_sum<N, T>(d2_sq, C);
  const float d2 = __fdividef(sqrt_approx(d2_sq * inv_denom), h0);
  const float h1 = (static_cast<double>(d1) <= 1e-15 && static_cast<double>(d2) <= 1e-15)
                       ? fmaxf(1e-6f, h0 * 1e-3f)
                       : __powf(__fdividef(0.01f, fmaxf(d1, d2)), 0.2f);
  float hm = 100.0f * h0;
  if (h1 < hm) hm = h1;
  if (P.max_dt < hm) hm = P.max_dt;
  s.h = hm;
  return true;
}

// A sim that stops in thread_attempt is written out later, by the persistent
// loop's finalize_pending, when its warp next refills: the warp's idle threads
// then run the FP64 finalize together instead of one at a time, while the other
// threads of the warp wait (CH4: 2.7 % faster, C2H6-like two threads per sim 4 %).
// Until then the per-step rejection counter and the stop threshold, no longer
// needed, hold the status and the final potential energy.
template <int N, int MODE, int T>
__device__ __forceinline__ void mark_finished(ThreadSim<N, MODE, T>& s, int status,
                                              typename ThreadSim<N, MODE, T>::Acc pe_final) {
  s.rej_in_step = static_cast<uint32_t>(status);
  s.pe_stop = pe_final;
}
template <int N, int MODE, int T, int F>
__device__ __forceinline__ void finalize_pending(const ThreadSim<N, MODE, T>& s, const RunParams& P,
                                                 const FixedMol& M, const MixedIn& X, const SimConsts<N, T>& C,
                                                 const float4* ks) {
  thread_finalize<N, MODE, T, F>(s, static_cast<int>(s.rej_in_step), static_cast<double>(s.pe_stop), P, M, X, C,
                                 ks);
}

// One DP5(4) attempt (src/integrators.cpp:83-146) plus, on acceptance, the
// driver's stop test (src/driver.cpp:19-30). `ks` is this thread's first stage
// chunk in shared memory; chunk c of stage slot l is ks[(l * NC + c) * B], B =
// sim_block<N, T>(), so every slot offset is an immediate.
// Returns false once the sim is finished (mark_finished).
template <int N, int MODE, int T, int F>
__device__ __forceinline__ bool thread_attempt(ThreadSim<N, MODE, T>& s, const RunParams& P, const FixedMol& M,
                                               const MixedIn& X, const SimConsts<N, T>& C, float4* ks) {
  using S = ThreadSim<N, MODE, T>;
  using Acc = typename S::Acc;
  constexpr int NC = SimShape<N, T>::NC;
  constexpr int NP = SimShape<N, T>::NP;
  constexpr int NF = SimShape<N, T>::NF;
  constexpr int B = sim_block<N, T>();
  const float hh = (P.max_dt < s.h) ? P.max_dt : s.h;  // std::min(h_, max_dt)

  // Stages 2..6: x_s = x + (c_s h) v + h^2 sum_l abar_sl k_l; k_s = a(x_s)
  // into slot s - 2.
  const float hh2 = hh * hh;
  float2 xs[NP], a[NP];
  {
    Acc no_pe = Acc(0);
#pragma unroll 1
    for (int si = 1; si <= 5; ++si) {
      // x + (c_s h) v first, then each stage's h^2 abar_sl k_l added on
      // (stage 2 has no k term)
      const float chh = c_c[si + 1] * hh;
#pragma unroll
      for (int p = 0; p < NP; ++p) xs[p] = pfma<NF>(p, bcast(chh), s.v[p], s.x[p]);
      if (si > 1) {
        const float a1 = c_abar[si + 1][1] * hh2;
        const float4* k1 = ks + s.k1s * NC * B;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const float4 q = k1[c * B];
          xs[2 * c] = pfma<NF>(2 * c, bcast(a1), make_float2(q.x, q.y), xs[2 * c]);
          xs[2 * c + 1] = pfma<NF>(2 * c + 1, bcast(a1), make_float2(q.z, q.w), xs[2 * c + 1]);
        }
      }
#pragma unroll 1
      for (int l = 1; l + 1 < si; ++l) {
        const float al = c_abar[si + 1][l + 1] * hh2;
        const float4* kl = ks + (l - 1) * NC * B;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const float4 q = kl[c * B];
          xs[2 * c] = pfma<NF>(2 * c, bcast(al), make_float2(q.x, q.y), xs[2 * c]);
          xs[2 * c + 1] = pfma<NF>(2 * c + 1, bcast(al), make_float2(q.z, q.w), xs[2 * c + 1]);
        }
      }
      sim_forces<N, T, Acc>(xs, a, M, C, false, no_pe);
      float4* out = ks + (si - 1) * NC * B;
#pragma unroll
      for (int c = 0; c < NC; ++c)
        out[c * B] = make_float4(a[2 * c].x, a[2 * c].y, a[2 * c + 1].x, a[2 * c + 1].y);
    }
  }

  // Stage 7 (row = 5th-order weights, c_7 = 1): x_new, and FSAL k7 with the
  // potential energy of x_new for the stop test.
  Acc pe_new = Acc(0);
  {
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      // one chunk's k2..k6 at a time keeps the stage-7 sums' live range short
      const float4 q1 = ks[(s.k1s * NC + (p >> 1)) * B];
      float2 sum = pmul<NF>(p, bcast(c_abar[7][1]), (p & 1) ? make_float2(q1.z, q1.w) : make_float2(q1.x, q1.y));
#pragma unroll
      for (int l = 1; l < 6; ++l) {
        const float4 q = ks[((l - 1) * NC + (p >> 1)) * B];
        sum = pfma<NF>(p, bcast(c_abar[7][l + 1]), (p & 1) ? make_float2(q.z, q.w) : make_float2(q.x, q.y), sum);
      }
      if (S::kKahan) {  // compensated update; the new compensation goes to the other cx slot
        const float2 inc = pfma<NF>(p, bcast(hh2), sum, pmul<NF>(p, bcast(hh), s.v[p]));
        const float4 qc = ks[(s.cxs * NC + (p >> 1)) * B];
        const float2 y = pfma<NF>(p, bcast(-1.0f), (p & 1) ? make_float2(qc.z, qc.w) : make_float2(qc.x, qc.y), inc);
        xs[p] = padd<NF>(p, s.x[p], y);
        const float2 cn = pfma<NF>(p, bcast(-1.0f), y, pfma<NF>(p, bcast(-1.0f), s.x[p], xs[p]));
        reinterpret_cast<float2*>(ks + ((15 - s.cxs) * NC + (p >> 1)) * B)[p & 1] = cn;
      } else {
        xs[p] = pfma<NF>(p, bcast(hh2), sum, pfma<NF>(p, bcast(hh), s.v[p], s.x[p]));  // c_7 = 1
      }
    }
    sim_forces<N, T, Acc>(xs, a, M, C, true, pe_new);
    pe_new = sim_sum<N, T>(pe_new, C);
#pragma unroll
    for (int c = 0; c < NC; ++c)
      ks[((11 - s.k1s) * NC + c) * B] = make_float4(a[2 * c].x, a[2 * c].y, a[2 * c + 1].x, a[2 * c + 1].y);
  }

  // x_new = xs. Velocity update and error estimate, one chunk at a time (stage
  // slots 0..4 hold k2..k6, slot 5 k7): v_new = v + h sum b_l k_l, position
  // error h^2 sum ebar_l k_l, velocity error h sum E_l k_l (b_2 = E_2 = 0).
  float2 vn[NP];
  float2 err2 = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    float4 q[6];
#pragma unroll
    for (int l = 0; l < 5; ++l) q[l] = ks[(l * NC + c) * B];
    q[5] = ks[((11 - s.k1s) * NC + c) * B];
    const float4 q1 = ks[(s.k1s * NC + c) * B];
#pragma unroll
    for (int hp = 0; hp < 2; ++hp) {
      const int p = 2 * c + hp;
      const float2 k1 = hp == 0 ? make_float2(q1.x, q1.y) : make_float2(q1.z, q1.w);
      float2 sv = pmul<NF>(p, bcast(c_b[1]), k1);
      float2 se = pmul<NF>(p, bcast(c_ebar[1]), k1);
      float2 sev = pmul<NF>(p, bcast(c_e[1]), k1);
#pragma unroll
      for (int l = 1; l < 6; ++l) {
        const float2 kl = hp == 0 ? make_float2(q[l - 1].x, q[l - 1].y) : make_float2(q[l - 1].z, q[l - 1].w);
        if (l != 1) sv = pfma<NF>(p, bcast(c_b[l + 1]), kl, sv);
        se = pfma<NF>(p, bcast(c_ebar[l + 1]), kl, se);
        if (l != 1) sev = pfma<NF>(p, bcast(c_e[l + 1]), kl, sev);
      }
      const float2 incv = pmul<NF>(p, bcast(hh), sv);
      if (S::kKahan) {  // compensated update; the new compensation goes to the other cv slot
        const float4 qc = ks[(s.cvs * NC + c) * B];
        const float2 y = pfma<NF>(p, bcast(-1.0f), hp == 0 ? make_float2(qc.x, qc.y) : make_float2(qc.z, qc.w), incv);
        vn[p] = padd<NF>(p, s.v[p], y);
        const float2 cn = pfma<NF>(p, bcast(-1.0f), y, pfma<NF>(p, bcast(-1.0f), s.v[p], vn[p]));
        reinterpret_cast<float2*>(ks + ((19 - s.cvs) * NC + c) * B)[hp] = cn;
      } else {
        vn[p] = padd<NF>(p, s.v[p], incv);
      }
      const float2 ex = pmul<NF>(p, bcast(hh2), se);
      const float2 k7 = hp == 0 ? make_float2(q[5].x, q[5].y) : make_float2(q[5].z, q[5].w);
      const float2 ev = pmul<NF>(p, bcast(hh), pfma<NF>(p, bcast(c_e[7]), k7, sev));
      // Scaled errors e / (atol + rtol max(|y0|, |y1|)), both halves of the pair
      // at once; a zero-padded half is left out (its scale could be 0).
      if (2 * p + 1 < NF) {
        const float2 sx = __ffma2_rn(bcast(P.rtol),
                                     make_float2(fmaxf(fabsf(s.x[p].x), fabsf(xs[p].x)),
                                                 fmaxf(fabsf(s.x[p].y), fabsf(xs[p].y))),
                                     bcast(P.atol));
        const float2 sv2 = __ffma2_rn(bcast(P.rtol),
                                      make_float2(fmaxf(fabsf(s.v[p].x), fabsf(vn[p].x)),
                                                  fmaxf(fabsf(s.v[p].y), fabsf(vn[p].y))),
                                      bcast(P.atol));
        const float2 rx = __fmul2_rn(ex, make_float2(rcp_approx(sx.x), rcp_approx(sx.y)));
        const float2 rv = __fmul2_rn(ev, make_float2(rcp_approx(sv2.x), rcp_approx(sv2.y)));
        err2 = __ffma2_rn(rv, rv, __ffma2_rn(rx, rx, err2));
      } else if (2 * p < NF) {
        const float rx = ex.x * rcp_approx(fmaf(P.rtol, fmaxf(fabsf(s.x[p].x), fabsf(xs[p].x)), P.atol));
        const float rv = ev.x * rcp_approx(fmaf(P.rtol, fmaxf(fabsf(s.v[p].x), fabsf(vn[p].x)), P.atol));
        err2.x = fmaf(rv, rv, fmaf(rx, rx, err2.x));
      }
    }
  }
  // RMS norm squared: en <= 1 exactly when en^2 <= 1, and the controller's
  // en^-1/5 is (en^2)^-1/10, so no square root is taken.
  const float en2 = sim_sum<N, T>(err2.x + err2.y, C) * (1.0f / static_cast<float>(6 * N));
  if (en2 <= 1.0f) {
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      s.x[p] = xs[p];
      s.v[p] = vn[p];
    }
    s.k1s = 11 - s.k1s;  // k7 becomes k1 (FSAL)
    if (S::kKahan) {  // the new compensation terms become current
      s.cxs = 15 - s.cxs;
      s.cvs = 19 - s.cvs;
    }
    float factor = (en2 == 0.0f) ? kMaxFactor : fminf(kMaxFactor, kSafety * __powf(en2, 0.5f * kExponent));
    if (s.rej_once) factor = fminf(factor, 1.0f);
    const float hn = hh * factor;
    s.h = (P.max_dt < hn) ? P.max_dt : hn;
    s.t += static_cast<Acc>(hh);
    s.steps += 1u;
    s.rej_in_step = 0u;
    s.rej_once = false;
    int fin = -1;
    if (!(pe_new > s.pe_stop)) fin = CE_SIM_OK;
    else if (s.steps >= P.max_steps) fin = CE_SIM_MAX_STEPS;
    if (fin >= 0) {
      mark_finished(s, fin, pe_new);
      return false;
    }
    return true;
  }
  s.h = hh * fmaxf(kMinFactor, kSafety * __powf(en2, 0.5f * kExponent));
  s.rej_once = true;
  s.rejects += 1u;
  s.rej_in_step += 1u;
  if (s.rej_in_step > static_cast<uint32_t>(kMaxRejections)) {
    mark_finished(s, CE_SIM_REJECT_LIMIT, pe_new);
    return false;
  }
  return true;
}

// Streamed-run helpers (RunParams io_*).
__device__ __forceinline__ unsigned ld_acquire_sys(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Waits until chunk j's positions are in device memory. Bounded: about 4 s of
// 256 ns sleeps, or until the host raises io_abort or another wait has already
// run out (io_error); then io_error is set and false returned. Both words live
// in host memory, so they are read only every 1024th poll: thousands of waiting
// warps reading across PCIe at every poll starve the very copies they wait for.
static __device__ __noinline__ bool io_wait_input(const unsigned* ready, const unsigned* abort_flag, unsigned* error) {
  constexpr unsigned kMaxPolls = 1u << 24;
  for (unsigned i = 0; i < kMaxPolls; ++i) {
    if (ld_acquire_gpu(ready) != 0u) return true;  // device memory, written by a copy
    if ((i & 1023u) == 1023u && (ld_acquire_sys(abort_flag) != 0u || ld_acquire_sys(error) != 0u)) break;
    __nanosleep(256);
  }
  *reinterpret_cast<volatile unsigned*>(error) = 1u;
  __threadfence_system();
  return false;
}

// Counts the sims the warp's threads finished in this iteration (fin) toward
// their chunks (chunk = sim >> io_shift): the finishing lanes are grouped by
// chunk, and after a __syncwarp one lane per group fences (covering the
// outputs its group wrote) and adds the group's count; the count that
// completes a chunk raises its host flag. Warp-collective; one ballot per
// iteration when nothing finished.
template <int T>
__device__ __forceinline__ void io_count(const RunParams& P, bool fin, unsigned long long sim) {
  unsigned rem = __ballot_sync(0xffffffffu, fin);
  if (rem == 0u) return;
  const unsigned j = static_cast<unsigned>(sim >> P.io_shift);
  __syncwarp();
  while (rem != 0u) {
    const int l = __ffs(rem) - 1;
    const unsigned jl = __shfl_sync(0xffffffffu, j, l);
    const unsigned grp = __ballot_sync(0xffffffffu, fin && j == jl);
    rem &= ~grp;
    if ((threadIdx.x & 31u) == static_cast<unsigned>(l)) {
      __threadfence();
      const unsigned long long lo = static_cast<unsigned long long>(jl) << P.io_shift;
      const unsigned long long hi = lo + (1ull << P.io_shift) < P.S ? lo + (1ull << P.io_shift) : P.S;
      const unsigned long long add = static_cast<unsigned long long>(__popc(grp));
      if (atomicAdd(P.io_done + jl, add) + add == static_cast<unsigned long long>(T) * (hi - lo)) {
        __threadfence_system();
        *reinterpret_cast<volatile unsigned*>(P.io_host_done + jl) = 1u;
      }
    }
  }
}

// Persistent loop of the mixed-batch two-thread buckets: each warp keeps its
// sims busy by pulling sim indices from the bucket's work queue `cursor` over
// [0, count), mapped through perm (one warp-aggregated atomicAdd per refill),
// whenever at least `refill` of its 16 sims are idle (or all of them); a sim is
// one even/odd lane pair, whose lanes are always active or idle together. The
// sims stopped since the last refill are written out first (finalize_pending).
template <int N, int MODE, int T, int F>
__device__ __forceinline__ void sim_loop(const RunParams& P, const FixedMol& M, const MixedIn& X,
                                         unsigned long long* cursor, unsigned long long count, const uint32_t* perm,
                                         int refill) {
  static_assert(T == 2 && (F & kLoopMixed) != 0 && (F & kLoopIO) == 0, "the mixed-batch two-thread loop");
  extern __shared__ float4 ce_stage_slots[];
  ThreadSim<N, MODE, T> s;
  SimConsts<N, T> C;
  bool active = false;
  bool queue_empty = count == 0ull;
  const unsigned lane = threadIdx.x & 31u;
  C.half = static_cast<int>(lane & 1u);  // per-sim constants are loaded at each claim
  C.pmask = 3u << (lane & 30u);
  constexpr unsigned kSimLanes = 0x55555555u;  // one lane per sim
  const unsigned first = lane & ~1u;           // this sim's first lane
  const unsigned lt_mask = (1u << first) - 1u;
  float4* ks = ce_stage_slots + threadIdx.x;
  const int B = static_cast<int>(blockDim.x);
  bool pending = false;  // this thread's stopped sim is not yet written out
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    const unsigned idle_s = idle & kSimLanes;
    const bool claim = !queue_empty && idle != 0u && (idle == 0xffffffffu || __popc(idle_s) >= refill);
    if ((claim || queue_empty) && pending) {
      finalize_pending<N, MODE, T, F>(s, P, M, X, C, ks);
      pending = false;
    }
    if (claim) {
      const int cnt = __popc(idle_s);
      const int leader = __ffs(idle_s) - 1;
      unsigned long long base = 0ull;
      if (static_cast<int>(lane) == leader) base = atomicAdd(cursor, static_cast<unsigned long long>(cnt));
      base = __shfl_sync(0xffffffffu, base, leader);
      queue_empty = (base + static_cast<unsigned long long>(cnt) >= count);
      if (!active) {
        const unsigned long long k = base + static_cast<unsigned long long>(__popc(idle_s & lt_mask));
        if (k < count) active = thread_init<N, MODE, T, F>(s, static_cast<unsigned long long>(perm[k]), P, M, X, C, ks, B);
      }
    }
    if (!__any_sync(0xffffffffu, active)) {
      if (queue_empty) break;
      continue;
    }
    if (active) {
      active = thread_attempt<N, MODE, T, F>(s, P, M, X, C, ks);
      pending = !active;
    }
  }
}

// Persistent loop of the fixed-molecule kernels: each warp pulls sim indices from
// the work queue P.cursor over [0, P.S) (one warp-aggregated atomicAdd per
// refill) whenever at least P.refill_threshold of its sims are idle (or all of
// them); a sim is one lane (T = 1) or one even/odd lane pair (T = 2). The sims
// stopped since the last refill are written out first (finalize_pending). With
// kLoopIO the claimed sims' inputs are awaited (io_wait_input) and written-out
// sims counted (io_count). Kept apart from sim_loop: the same loop with the
// queue passed as arguments ran the CH4 kernel 0.5 % slower.
template <int N, int MODE, int T, int F>
__device__ __forceinline__ void fixed_loop(const RunParams& P, const FixedMol& M) {
  constexpr bool IO = (F & kLoopIO) != 0;
  extern __shared__ float4 ce_stage_slots[];
  const MixedIn X{};
  ThreadSim<N, MODE, T> s;
  SimConsts<N, T> C;
  bool active = false;
  bool queue_empty = false;
  const unsigned lane = threadIdx.x & 31u;
  if constexpr (T == 2) load_pair_consts<N>(C, M, lane);
  constexpr unsigned kSimLanes = T == 2 ? 0x55555555u : 0xffffffffu;  // one lane per sim
  const unsigned first = T == 2 ? (lane & ~1u) : lane;                // this sim's first lane
  const unsigned lt_mask = (1u << first) - 1u;
  float4* ks = ce_stage_slots + threadIdx.x;
  const int B = static_cast<int>(blockDim.x);
  unsigned io_known = 0u;  // IO: chunks [0, io_known) seen present by this warp
  bool pending = false;    // this thread's stopped sim is not yet written out
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    const unsigned idle_s = idle & kSimLanes;
    const bool claim = !queue_empty && idle != 0u && (idle == 0xffffffffu || __popc(idle_s) >= P.refill_threshold);
    if (claim || queue_empty) {  // warp-uniform: the stopped sims are written out together
      if (pending) finalize_pending<N, MODE, T, F>(s, P, M, X, C, ks);
      if constexpr (IO) io_count<T>(P, pending, s.sim);
      pending = false;
    }
    bool fin = false;  // IO: this thread's sim finished at its claim
    unsigned long long fin_sim = 0ull;
    if (claim) {
      const int cnt = __popc(idle_s);
      const int leader = __ffs(idle_s) - 1;
      unsigned long long base = 0ull;
      if (static_cast<int>(lane) == leader) base = atomicAdd(P.cursor, static_cast<unsigned long long>(cnt));
      base = __shfl_sync(0xffffffffu, base, leader);
      queue_empty = (base + static_cast<unsigned long long>(cnt) >= P.S);
      bool in_ok = true;
      if constexpr (IO) {
        if (base < P.S) {
          const unsigned long long last = (base + cnt < P.S ? base + cnt : P.S) - 1ull;
          const unsigned lc = static_cast<unsigned>(last >> P.io_shift);
          if (lc >= io_known) {
            if (static_cast<int>(lane) == leader) in_ok = io_wait_input(P.io_ready + lc, P.io_abort, P.io_error);
            in_ok = __shfl_sync(0xffffffffu, in_ok, leader);
            if (in_ok) io_known = lc + 1u;
          }
        }
      }
      if (!active) {
        const unsigned long long sim = base + static_cast<unsigned long long>(__popc(idle_s & lt_mask));
        if (sim < P.S) {
          if (in_ok) {
            active = thread_init<N, MODE, T, F>(s, sim, P, M, X, C, ks, B);
          } else if (P.status && lane == first) {
            P.status[sim] = static_cast<uint8_t>(CE_SIM_BAD_INPUT);
          }
          fin = !active;
          fin_sim = sim;
        }
      }
    }
    if constexpr (IO) io_count<T>(P, fin, fin_sim);
    if (!__any_sync(0xffffffffu, active)) {
      if (queue_empty) break;
      continue;
    }
    if (active) {
      active = thread_attempt<N, MODE, T, F>(s, P, M, X, C, ks);
      pending = !active;
    }
  }
}

// One thread per sim: thread_block(N) threads per block and
// thread_smem_bytes(N, thread_block(N), MODE) bytes of dynamic shared memory.
template <int N, int MODE>
__global__ void __launch_bounds__(thread_block(N), (thread_min_blocks<N, MODE>()))
    rk45_fixed_kernel(const RunParams P, const FixedMol M) {
  fixed_loop<N, MODE, 1, 0>(P, M);
}

// Two threads per sim (N >= 3): kPairBlock threads per block and
// pair_smem_bytes(N, MODE) bytes of dynamic shared memory.
template <int N, int MODE>
__global__ void __launch_bounds__(kPairBlock, (pair_min_blocks<N, MODE>()))
    rk45_pair_kernel(const RunParams P, const FixedMol M) {
  fixed_loop<N, MODE, 2, 0>(P, M);
}

// The same two kernels with streamed host-buffer I/O (RunParams io_*).
template <int N, int MODE>
__global__ void __launch_bounds__(thread_block(N), (thread_min_blocks<N, MODE>()))
    rk45_fixed_io_kernel(const RunParams P, const FixedMol M) {
  fixed_loop<N, MODE, 1, kLoopIO>(P, M);
}
template <int N, int MODE>
__global__ void __launch_bounds__(kPairBlock, (pair_min_blocks<N, MODE>()))
    rk45_pair_io_kernel(const RunParams P, const FixedMol M) {
  fixed_loop<N, MODE, 2, kLoopIO>(P, M);
}

// One size bucket of a mixed batch in the two-thread layout (the per-size
// schedule with mixed lanes_per_sim = 2), with saved / resumed integrator state
// (RunParams save_* / res_*); launched like rk45_pair_kernel.
template <int N, int MODE>
__global__ void __launch_bounds__(kPairBlock, (pair_min_blocks<N, MODE>()))
    rk45_pair_bucket_kernel(const RunParams P, const MixedIn X, const Buckets B) {
  const FixedMol none{};
  sim_loop<N, MODE, 2, kLoopMixed | kLoopState>(P, none, X, B.cursor + N, B.cnt[N], B.perm + B.off[N],
                                                P.refill_threshold);
}

using FixedKernelFn = void (*)(RunParams, FixedMol);
// One dispatch function per precision mode, defined in kernels_fixed.cu.
FixedKernelFn fixed_kernel_m0(int n);
FixedKernelFn fixed_kernel_m1(int n);
FixedKernelFn fixed_kernel_m2(int n);
FixedKernelFn fixed_kernel_m3(int n);
// Two-thread layout, N = 3..10 (nullptr otherwise).
FixedKernelFn pair_kernel_m0(int n);
FixedKernelFn pair_kernel_m1(int n);
FixedKernelFn pair_kernel_m2(int n);
FixedKernelFn pair_kernel_m3(int n);
// The streamed-I/O variants: pair = false for one thread per sim (N = 1..10),
// true for two threads per sim (N = 3..10).
FixedKernelFn io_kernel_m0(int n, bool pair);
FixedKernelFn io_kernel_m1(int n, bool pair);
FixedKernelFn io_kernel_m2(int n, bool pair);
FixedKernelFn io_kernel_m3(int n, bool pair);
// The mixed-batch two-thread bucket kernels, N = 3..10 (nullptr otherwise).
using PairBucketFn = void (*)(RunParams, MixedIn, Buckets);
PairBucketFn pair_bucket_kernel_m0(int n);
PairBucketFn pair_bucket_kernel_m1(int n);
PairBucketFn pair_bucket_kernel_m2(int n);
PairBucketFn pair_bucket_kernel_m3(int n);

}  // namespace ce
