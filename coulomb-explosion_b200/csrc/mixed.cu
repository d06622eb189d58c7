// mixed.cu -- mixed 2..10-atom batches, CUDA-graph capture and the autotuner
// (include/ce_gpu.h).
//
// The reference runs one molecule per BatchedRK45 (every lane shares the
// molecule, include/coulomb/batched_force.hpp:8-13); a mixed population takes
// one reference engine per molecule. Here one call integrates any mix: a
// device counting sort groups the sims by atom count (count -> scan -> scatter,
// three small kernels), then either one persistent launch walks the size
// buckets (CE_SCHEDULE_ONE_LAUNCH) or one launch per bucket runs them in
// sequence (CE_SCHEDULE_PER_SIZE). Everything is stream-ordered and allocates
// nothing once ce_reserve_mixed has sized the scratch, so it can be captured
// into a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "ce_gpu.h"
#include "engine.hpp"

namespace {

constexpr int kBins = 16;  // bin 0 = invalid atom count, bins 1..10 = atoms per sim

// Bucket tables at the head of the engine's mixed scratch (u64 each).
struct BucketTables {
  unsigned long long* cnt;     // [kBins]
  unsigned long long* off;     // [kBins]
  unsigned long long* fill;    // [kBins]
  unsigned long long* cursor;  // [kBins]
  uint32_t* perm;              // [S]
};

size_t mixed_scratch_bytes(uint64_t S) { return 4 * kBins * sizeof(unsigned long long) + S * sizeof(uint32_t); }

BucketTables tables_of(void* base) {
  auto* p = static_cast<unsigned long long*>(base);
  BucketTables t;
  t.cnt = p;
  t.off = p + kBins;
  t.fill = p + 2 * kBins;
  t.cursor = p + 3 * kBins;
  t.perm = reinterpret_cast<uint32_t*>(p + 4 * kBins);
  return t;
}

__device__ __forceinline__ int bin_of(uint8_t n) { return (n >= 1 && n <= CE_MAX_ATOMS) ? n : 0; }

__global__ void bucket_count_kernel(const uint8_t* __restrict__ n_per, uint64_t S, unsigned long long* cnt) {
  __shared__ unsigned int h[kBins];
  if (threadIdx.x < kBins) h[threadIdx.x] = 0u;
  __syncthreads();
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < S;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    atomicAdd(&h[bin_of(n_per[i])], 1u);
  __syncthreads();
  if (threadIdx.x < kBins && h[threadIdx.x]) atomicAdd(&cnt[threadIdx.x], static_cast<unsigned long long>(h[threadIdx.x]));
}

__global__ void bucket_scan_kernel(const unsigned long long* cnt, unsigned long long* off, unsigned long long* fill,
                                   unsigned long long* cursor) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned long long acc = 0ull;
  for (int b = 0; b < kBins; ++b) {
    off[b] = acc;
    acc += cnt[b];
    fill[b] = 0ull;
    cursor[b] = 0ull;
  }
}

// Scatter sim indices into their bucket (order inside a bucket is irrelevant:
// every sim is integrated independently). Sims with one atom (no pair, PE = 0,
// converged at rest) and sims with an invalid atom count are written out here.
__global__ void bucket_scatter_kernel(const uint8_t* __restrict__ n_per, uint64_t S, const unsigned long long* off,
                                      unsigned long long* fill, uint32_t* perm, ce::RunParams P) {
  __shared__ unsigned int h[kBins];
  __shared__ unsigned long long b[kBins];
  for (uint64_t t0 = blockIdx.x * static_cast<uint64_t>(blockDim.x); t0 < S;
       t0 += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    if (threadIdx.x < kBins) h[threadIdx.x] = 0u;
    __syncthreads();
    const uint64_t i = t0 + threadIdx.x;
    int bin = -1;
    unsigned int r = 0u;
    if (i < S) {
      bin = bin_of(n_per[i]);
      r = atomicAdd(&h[bin], 1u);
    }
    __syncthreads();
    if (threadIdx.x < kBins && h[threadIdx.x]) b[threadIdx.x] = atomicAdd(&fill[threadIdx.x], static_cast<unsigned long long>(h[threadIdx.x]));
    __syncthreads();
    if (bin >= 2) {
      perm[off[bin] + b[bin] + r] = static_cast<uint32_t>(i);
    } else if (bin >= 0 && !(P.skip_empty && n_per[i] == 0)) {
      float* m = P.momenta + i * (3ull * ce::kMixedStride);
      for (int c = 0; c < 3 * ce::kMixedStride; ++c) m[c] = 0.0f;
      if (P.ker) P.ker[i] = 0.0;
      if (P.steps) P.steps[i] = 0u;
      if (P.status) P.status[i] = bin == 1 ? static_cast<uint8_t>(CE_SIM_OK) : static_cast<uint8_t>(CE_SIM_BAD_INPUT);
      if (P.rejects) P.rejects[i] = 0u;
      if (P.t_final) P.t_final[i] = 0.0;
      if (P.pe_final) P.pe_final[i] = 0.0;
      if (P.ke_before) P.ke_before[i] = 0.0;
      if (P.e0) P.e0[i] = 0.0;
      if (P.positions) {
        float* xp = P.positions + i * (3ull * ce::kMixedStride);
        const float* x0 = P.pos + i * (3ull * ce::kMixedStride);
        for (int c = 0; c < 3 * ce::kMixedStride; ++c) xp[c] = bin == 1 ? x0[c] : 0.0f;
      }
      if (P.save_h) {  // saved state of a sim that needs no integration: restart from rest
        const float* x0 = P.pos + i * (3ull * ce::kMixedStride);
        for (int c = 0; c < 3 * ce::kMixedStride; ++c) {
          P.save_pos[i * (3ull * ce::kMixedStride) + c] = bin == 1 ? x0[c] : 0.0f;
          P.save_vel[i * (3ull * ce::kMixedStride) + c] = 0.0f;
        }
        if (P.save_comp)
          for (int c = 0; c < 6 * ce::kMixedStride; ++c) P.save_comp[i * (6ull * ce::kMixedStride) + c] = 0.0f;
        P.save_h[i] = 0.0f;
        P.save_t[i] = 0.0;
        P.save_steps[i] = 0u;
        P.save_rejects[i] = 0u;
        P.save_e0[i] = 0.0;
      }
    }
    __syncthreads();
  }
}

// Launch shape of the mixed path; refill_threshold stays 0 ("per size") unless
// set by the caller or the autotuner.
ce_tuning mixed_tuning(const ce_engine* e) {
  ce_tuning t = e->tuning;
  const ce_tuned_entry& a = e->tuned_mixed;
  if (t.block_threads == 0) t.block_threads = a.valid && a.t.block_threads ? a.t.block_threads : 128;
  if (t.blocks_per_sm == 0 && a.valid) t.blocks_per_sm = a.t.blocks_per_sm;
  if (t.refill_threshold == 0 && a.valid) t.refill_threshold = a.t.refill_threshold;
  if (t.lanes_per_sim == 0 && a.valid) t.lanes_per_sim = a.t.lanes_per_sim;
  return t;
}

// Whether the n-atom bucket runs two threads per sim (mixed lanes_per_sim = 2,
// 3 or more atoms) rather than one lane per atom.
bool pair_bucket(const ce_tuning& t, int n) { return t.lanes_per_sim == 2 && n >= 3; }

// Dynamic shared memory above the default 48 KB, and all of the SM's unified
// L1 / shared storage as shared memory, for a kernel that takes `smem` bytes.
int prepare_smem(ce_engine* e, const void* fn, size_t smem) {
  if (smem == 0) return CE_OK;
  cudaError_t st = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaFuncSetAttribute(max dynamic shared memory)");
  st = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaFuncSetAttribute(shared memory carveout)");
  return CE_OK;
}

int check_mixed_args(ce_engine* e, uint64_t S, const ce_mixed_batch* in, double k, const ce_run_config* cfg,
                     const ce_outputs* out) {
  int rc = ce::check_config(e, cfg);
  if (rc != CE_OK) return rc;
  if (S >= (1ull << 32)) return ce::fail(e, CE_ERR_INVALID, "ce_run_mixed: S must be below 2^32");
  if (S == 0) return CE_OK;
  if (!in || !in->n_atoms || !in->mass_me || !in->charge || !in->pos)
    return ce::fail(e, CE_ERR_INVALID, "ce_run_mixed: n_atoms, mass_me, charge and pos are required");
  if (!out || !out->momenta) return ce::fail(e, CE_ERR_INVALID, "ce_run_mixed: out->momenta is required");
  if (!std::isfinite(k)) return ce::fail(e, CE_ERR_INVALID, "ce_run_mixed: non-finite Coulomb constant");
  return CE_OK;
}

}  // namespace

struct ce_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = 0;
};

namespace {
// The side stream and events of CE_SCHEDULE_OVERLAP, created once (outside any capture).
int ensure_overlap_stream(ce_engine* e) {
  if (e->s_mix2) return CE_OK;
  cudaError_t st;
  if ((st = cudaStreamCreateWithFlags(&e->s_mix2, cudaStreamNonBlocking)) != cudaSuccess ||
      (st = cudaEventCreateWithFlags(&e->ev_mix_fork, cudaEventDisableTiming)) != cudaSuccess ||
      (st = cudaEventCreateWithFlags(&e->ev_mix_join, cudaEventDisableTiming)) != cudaSuccess)
    return ce::cuda_fail(e, st, "overlap schedule stream");
  return CE_OK;
}
}  // namespace

extern "C" {

int ce_reserve_mixed(ce_engine* e, uint64_t S) {
  if (!e) return CE_ERR_INVALID;
  if (S >= (1ull << 32)) return ce::fail(e, CE_ERR_INVALID, "ce_reserve_mixed: S must be below 2^32");
  cudaError_t st = cudaSetDevice(e->device);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaSetDevice");
  int rc = ensure_overlap_stream(e);
  if (rc != CE_OK) return rc;
  const size_t need = mixed_scratch_bytes(S);
  if (need <= e->mixed_bytes) return CE_OK;
  if (e->d_mixed) cudaFree(e->d_mixed);
  e->d_mixed = nullptr;
  e->mixed_bytes = 0;
  st = cudaMalloc(&e->d_mixed, need);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaMalloc(mixed scratch)");
  e->mixed_bytes = need;
  return CE_OK;
}

int ce_run_mixed_device(ce_engine* e, uint64_t S, const ce_mixed_batch* in, double coulomb_k,
                        const ce_run_config* cfg, const ce_outputs* out, int schedule, void* stream) {
  return ce::run_mixed_device(e, S, in, coulomb_k, cfg, out, schedule, stream, false, nullptr, nullptr);
}

int ce_run_mixed_device_state(ce_engine* e, uint64_t S, const ce_mixed_batch* in, double coulomb_k,
                              const ce_run_config* cfg, const ce_sim_state* resume, const ce_sim_state* save,
                              const ce_outputs* out, int schedule, void* stream) {
  return ce::run_mixed_device(e, S, in, coulomb_k, cfg, out, schedule, stream, false, resume, save);
}

}  // extern "C"

namespace ce {

int run_mixed_device(ce_engine* e, uint64_t S, const ce_mixed_batch* in, double coulomb_k, const ce_run_config* cfg,
                     const ce_outputs* out, int schedule, void* stream, bool skip_empty, const ce_sim_state* resume,
                     const ce_sim_state* save) {
  if (!e) return CE_ERR_INVALID;
  e->last_launches = 0;
  int rc = check_mixed_args(e, S, in, coulomb_k, cfg, out);
  if (rc != CE_OK || S == 0) return rc;
  const bool kahan = (cfg->precision_mode & CE_PREC_KAHAN) != 0;
  for (const ce_sim_state* st : {resume, save})
    if (st && (!st->positions || !st->velocities || !st->h || !st->t || !st->steps || !st->rejects || !st->e0 ||
               (kahan && !st->comp)))
      return ce::fail(e, CE_ERR_INVALID, "ce_run_mixed_device_state: a state pointer is NULL");
  if (schedule != CE_SCHEDULE_ONE_LAUNCH && schedule != CE_SCHEDULE_PER_SIZE && schedule != CE_SCHEDULE_OVERLAP)
    return ce::fail(e, CE_ERR_INVALID, "ce_run_mixed: unknown schedule");
  const ce_tuning t = mixed_tuning(e);
  // Saving and resuming integrator state is built into the per-size kernels only
  // (in the one-launch kernel the extra registers cost 6 %), and so are the
  // two-thread buckets (lanes_per_sim = 2).
  if ((resume || save || t.lanes_per_sim == 2) && schedule == CE_SCHEDULE_ONE_LAUNCH) schedule = CE_SCHEDULE_PER_SIZE;
  cudaError_t st = cudaSetDevice(e->device);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaSetDevice");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (mixed_scratch_bytes(S) > e->mixed_bytes || !e->s_mix2) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (s && cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone)
      return ce::fail(e, CE_ERR_STATE, "ce_run_mixed: scratch too small during graph capture (ce_reserve_mixed first)");
    rc = ce_reserve_mixed(e, S);
    if (rc != CE_OK) return rc;
  }
  const BucketTables T = tables_of(e->d_mixed);

  ce::RunParams P{};
  ce::fill_run_params(P, cfg, out, t.refill_threshold);  // 0: each size's default
  P.skip_empty = skip_empty ? 1 : 0;
  P.pos = in->pos;
  P.cursor = nullptr;
  if (save) {
    P.save_pos = save->positions;
    P.save_vel = save->velocities;
    P.save_h = save->h;
    P.save_t = save->t;
    P.save_steps = save->steps;
    P.save_rejects = save->rejects;
    P.save_e0 = save->e0;
    P.save_comp = save->comp;
  }
  if (resume) {
    P.res_pos = resume->positions;
    P.res_vel = resume->velocities;
    P.res_h = resume->h;
    P.res_t = resume->t;
    P.res_steps = resume->steps;
    P.res_rejects = resume->rejects;
    P.res_e0 = resume->e0;
    P.res_comp = resume->comp;
  }
  P.S = S;
  ce::MixedIn X{in->n_atoms, in->mass_me, in->charge, coulomb_k};
  ce::Buckets B{T.perm, T.off, T.cnt, T.cursor};

  const int sort_block = 256;
  const unsigned sort_grid =
      static_cast<unsigned>(std::min<uint64_t>((S + sort_block - 1) / sort_block, static_cast<uint64_t>(e->sms) * 8));
  st = cudaMemsetAsync(T.cnt, 0, kBins * sizeof(unsigned long long), s);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaMemsetAsync(bucket counts)");
  bucket_count_kernel<<<sort_grid, sort_block, 0, s>>>(in->n_atoms, S, T.cnt);
  bucket_scan_kernel<<<1, 32, 0, s>>>(T.cnt, T.off, T.fill, T.cursor);
  bucket_scatter_kernel<<<sort_grid, sort_block, 0, s>>>(in->n_atoms, S, T.off, T.fill, T.perm, P);
  int launches = 3;

  const int block = std::min(t.block_threads, ce::kAtomMaxBlock);
  if (schedule == CE_SCHEDULE_ONE_LAUNCH) {
    const ce::MixedKernelFn fn = ce::select_mixed_kernel(0, cfg->precision_mode);
    int per_sm = t.blocks_per_sm;
    if (per_sm == 0) {
      st = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, 0);
      if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
      if (per_sm < 1) per_sm = 1;
    }
    // Enough groups for the smallest molecules, never more than one wave.
    const uint64_t sims_per_block = static_cast<uint64_t>(block / 32) * (32 / 2);
    const uint64_t grid = std::min<uint64_t>(static_cast<uint64_t>(e->sms) * per_sm, (S + sims_per_block - 1) / sims_per_block);
    fn<<<static_cast<unsigned>(std::max<uint64_t>(grid, 1)), block, 0, s>>>(P, X, B);
    ++launches;
  } else {
    // Per size, 10 atoms down to 2; with CE_SCHEDULE_OVERLAP the launches
    // alternate between the call's stream and the engine's side stream (forked
    // after the sort, joined at the end), so a bucket's blocks take over SMs as
    // the previous bucket's last blocks retire.
    const bool overlap = schedule == CE_SCHEDULE_OVERLAP;
    if (overlap) {
      if ((st = cudaEventRecord(e->ev_mix_fork, s)) != cudaSuccess ||
          (st = cudaStreamWaitEvent(e->s_mix2, e->ev_mix_fork, 0)) != cudaSuccess)
        return ce::cuda_fail(e, st, "overlap schedule fork");
    }
    for (int n = CE_MAX_ATOMS; n >= 2; --n) {
      const cudaStream_t sn = (overlap && (n & 1)) ? e->s_mix2 : s;
      const bool pair = pair_bucket(t, n);
      const ce::MixedKernelFn fn = pair ? ce::select_pair_bucket_kernel(n, cfg->precision_mode)
                                        : ce::select_mixed_kernel(n, cfg->precision_mode);
      const int bn = pair ? ce::kPairBlock : block;
      const size_t smem = pair ? ce::pair_smem_bytes(n, cfg->precision_mode) : 0;
      rc = prepare_smem(e, reinterpret_cast<const void*>(fn), smem);
      if (rc != CE_OK) return rc;
      int per_sm = t.blocks_per_sm;
      if (per_sm == 0) {
        st = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, bn, smem);
        if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        if (per_sm < 1) per_sm = 1;
      }
      const uint64_t sims_per_block =
          pair ? static_cast<uint64_t>(bn / 2) : static_cast<uint64_t>(bn / 32) * (32 / n);
      const uint64_t grid = std::min<uint64_t>(static_cast<uint64_t>(e->sms) * per_sm, (S + sims_per_block - 1) / sims_per_block);
      ce::RunParams Pn = P;
      if (t.refill_threshold == 0) Pn.refill_threshold = ce::default_refill(n, pair ? 2 : n);
      fn<<<static_cast<unsigned>(std::max<uint64_t>(grid, 1)), bn, smem, sn>>>(Pn, X, B);
      ++launches;
    }
    if (overlap) {
      if ((st = cudaEventRecord(e->ev_mix_join, e->s_mix2)) != cudaSuccess ||
          (st = cudaStreamWaitEvent(s, e->ev_mix_join, 0)) != cudaSuccess)
        return ce::cuda_fail(e, st, "overlap schedule join");
    }
  }
  st = cudaGetLastError();
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "mixed kernel launch");
  e->last_launches = launches;
  return CE_OK;
}

}  // namespace ce

extern "C" {

// Host-buffer path, pipelined like ce_run: the batch is cut into up to 8 chunks
// that alternate between two device slots; chunk k's inputs go up on a copy-in
// stream while chunk k-1 integrates on the engine stream and chunk k-2's results
// come down on a copy-out stream (with pinned host buffers the copies overlap the
// kernels). The chunks integrate one after another on the engine stream, since
// they share the engine's bucket-sort scratch.
int ce_run_mixed(ce_engine* e, uint64_t S, const ce_mixed_batch* in, double coulomb_k, const ce_run_config* cfg,
                 const ce_outputs* out) {
  if (!e) return CE_ERR_INVALID;
  int rc = check_mixed_args(e, S, in, coulomb_k, cfg, out);
  if (rc != CE_OK || S == 0) return rc;
  cudaError_t st = cudaSetDevice(e->device);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaSetDevice");
  rc = ce::ensure_pipeline(e);
  if (rc != CE_OK) return rc;
  uint64_t bnd[17], C = 0;
  const uint64_t nchunks = ce::chunk_bounds(S, 1ull << 17, 8, bnd, &C);
  rc = ce_reserve_mixed(e, C);  // before any chunk is queued: a reallocation synchronises
  if (rc != CE_OK) return rc;

  const size_t A = CE_MAX_ATOMS;
  auto al = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
  const size_t sizes[] = {al(C),                              // n_atoms
                          al(C * A * sizeof(double)),         // mass
                          al(C * A * sizeof(double)),         // charge
                          al(C * A * 3 * sizeof(float)),      // pos
                          al(C * A * 3 * sizeof(float)),      // momenta
                          al(C * sizeof(double)) * 5,         // ker, t_final, pe_final, ke_before, e0
                          al(C * sizeof(uint32_t)) * 2,       // steps, rejects
                          al(C),                              // status
                          al(C * A * 3 * sizeof(float))};     // positions at termination
  size_t slot_bytes = 0;
  for (size_t b : sizes) slot_bytes += b;
  const int nslots = nchunks > 1 ? 2 : 1;
  const size_t total = slot_bytes * nslots;
  if (total > e->arena_bytes) {
    cudaDeviceSynchronize();
    if (e->d_arena) cudaFree(e->d_arena);
    e->d_arena = nullptr;
    e->arena_bytes = 0;
    st = cudaMalloc(&e->d_arena, total);
    if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaMalloc(arena)");
    e->arena_bytes = total;
  }
  struct Slot {
    char *n, *m, *q, *x;
    ce_outputs d;
  } slots[2];
  const size_t bd = al(C * sizeof(double)), bu = al(C * sizeof(uint32_t));
  for (int k = 0; k < nslots; ++k) {
    char* p = static_cast<char*>(e->d_arena) + k * slot_bytes;
    Slot& sl = slots[k];
    sl.n = p;
    p += sizes[0];
    sl.m = p;
    p += sizes[1];
    sl.q = p;
    p += sizes[2];
    sl.x = p;
    p += sizes[3];
    sl.d = ce_outputs{};
    sl.d.momenta = reinterpret_cast<float*>(p);
    p += sizes[4];
    sl.d.ker = out->ker ? reinterpret_cast<double*>(p) : nullptr;
    sl.d.t_final = out->t_final ? reinterpret_cast<double*>(p + bd) : nullptr;
    sl.d.pe_final = out->pe_final ? reinterpret_cast<double*>(p + 2 * bd) : nullptr;
    sl.d.ke_before = out->ke_before ? reinterpret_cast<double*>(p + 3 * bd) : nullptr;
    sl.d.e0 = out->e0 ? reinterpret_cast<double*>(p + 4 * bd) : nullptr;
    p += sizes[5];
    sl.d.steps = out->steps ? reinterpret_cast<uint32_t*>(p) : nullptr;
    sl.d.rejects = out->rejects ? reinterpret_cast<uint32_t*>(p + bu) : nullptr;
    p += sizes[6];
    sl.d.status = out->status ? reinterpret_cast<uint8_t*>(p) : nullptr;
    p += sizes[7];
    sl.d.positions = out->positions ? reinterpret_cast<float*>(p) : nullptr;
  }

  struct Copy {
    void* dst;
    const void* src;
    size_t bytes;
  };
  int launches = 0;
  for (uint64_t k = 0; k < nchunks; ++k) {
    const uint64_t s0 = bnd[k], Sk = bnd[k + 1] - bnd[k];
    if (Sk == 0) continue;
    const int si = static_cast<int>(k % nslots);
    Slot& sl = slots[si];
    // inputs up once the slot's previous chunk has been integrated
    if (k >= 2 && (rc = ce::wait_on(e, e->s_in, e->ev_computed[si])) != CE_OK) return rc;
    const Copy h2d[] = {{sl.n, in->n_atoms + s0, Sk},
                        {sl.m, in->mass_me + s0 * A, Sk * A * sizeof(double)},
                        {sl.q, in->charge + s0 * A, Sk * A * sizeof(double)},
                        {sl.x, in->pos + s0 * A * 3, Sk * A * 3 * sizeof(float)}};
    for (const Copy& c : h2d) {
      st = cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyHostToDevice, e->s_in);
      if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaMemcpyAsync(H2D)");
    }
    if ((rc = ce::record(e, e->ev_loaded[si], e->s_in)) != CE_OK) return rc;
    // integrate once the inputs are in and the slot's previous results are out
    if ((rc = ce::wait_on(e, e->stream, e->ev_loaded[si])) != CE_OK) return rc;
    if (k >= 2 && (rc = ce::wait_on(e, e->stream, e->ev_copied[si])) != CE_OK) return rc;
    // the kernels write atoms < n only: clear the rows, so the padding that comes
    // back is zero and not an earlier chunk's
    st = cudaMemsetAsync(sl.d.momenta, 0, Sk * A * 3 * sizeof(float), e->stream);
    if (st == cudaSuccess && sl.d.positions)
      st = cudaMemsetAsync(sl.d.positions, 0, Sk * A * 3 * sizeof(float), e->stream);
    if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaMemsetAsync(rows)");
    const ce_mixed_batch d_in{reinterpret_cast<const uint8_t*>(sl.n), reinterpret_cast<const double*>(sl.m),
                              reinterpret_cast<const double*>(sl.q), reinterpret_cast<const float*>(sl.x)};
    rc = ce_run_mixed_device(e, Sk, &d_in, coulomb_k, cfg, &sl.d, e->tuned_schedule, e->stream);
    if (rc != CE_OK) return rc;
    launches += e->last_launches;
    if ((rc = ce::record(e, e->ev_computed[si], e->stream)) != CE_OK) return rc;
    // results down
    if ((rc = ce::wait_on(e, e->s_out, e->ev_computed[si])) != CE_OK) return rc;
    const Copy d2h[] = {
        {out->momenta + s0 * A * 3, sl.d.momenta, Sk * A * 3 * sizeof(float)},
        {out->ker ? out->ker + s0 : nullptr, sl.d.ker, Sk * sizeof(double)},
        {out->t_final ? out->t_final + s0 : nullptr, sl.d.t_final, Sk * sizeof(double)},
        {out->pe_final ? out->pe_final + s0 : nullptr, sl.d.pe_final, Sk * sizeof(double)},
        {out->ke_before ? out->ke_before + s0 : nullptr, sl.d.ke_before, Sk * sizeof(double)},
        {out->steps ? out->steps + s0 : nullptr, sl.d.steps, Sk * sizeof(uint32_t)},
        {out->rejects ? out->rejects + s0 : nullptr, sl.d.rejects, Sk * sizeof(uint32_t)},
        {out->status ? out->status + s0 : nullptr, sl.d.status, Sk},
        {out->positions ? out->positions + s0 * A * 3 : nullptr, sl.d.positions, Sk * A * 3 * sizeof(float)},
        {out->e0 ? out->e0 + s0 : nullptr, sl.d.e0, Sk * sizeof(double)}};
    for (const Copy& c : d2h) {
      if (!c.dst) continue;
      st = cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, e->s_out);
      if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaMemcpyAsync(D2H)");
    }
    if ((rc = ce::record(e, e->ev_copied[si], e->s_out)) != CE_OK) return rc;
  }
  e->last_launches = launches;
  st = cudaStreamSynchronize(e->s_out);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e->stream);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaStreamSynchronize");
  return CE_OK;
}

// ---- CUDA graphs ----------------------------------------------------------

int ce_graph_begin(ce_engine* e, void* stream) {
  if (!e) return CE_ERR_INVALID;
  if (!stream) return ce::fail(e, CE_ERR_INVALID, "ce_graph_begin: capture needs a non-default stream");
  cudaError_t st = cudaSetDevice(e->device);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaSetDevice");
  st = cudaStreamBeginCapture(static_cast<cudaStream_t>(stream), cudaStreamCaptureModeThreadLocal);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaStreamBeginCapture");
  return CE_OK;
}

int ce_graph_end(ce_engine* e, void* stream, ce_graph** out) {
  if (!e || !out) return CE_ERR_INVALID;
  *out = nullptr;
  cudaGraph_t g = nullptr;
  cudaError_t st = cudaStreamEndCapture(static_cast<cudaStream_t>(stream), &g);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaStreamEndCapture");
  cudaGraphExec_t x = nullptr;
  st = cudaGraphInstantiate(&x, g, 0);
  if (st != cudaSuccess) {
    cudaGraphDestroy(g);
    return ce::cuda_fail(e, st, "cudaGraphInstantiate");
  }
  ce_graph* h = new ce_graph();
  h->graph = g;
  h->exec = x;
  h->device = e->device;
  *out = h;
  return CE_OK;
}

int ce_graph_launch(ce_graph* g, void* stream) {
  if (!g) return CE_ERR_INVALID;
  if (cudaSetDevice(g->device) != cudaSuccess) return CE_ERR_CUDA;
  return cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream)) == cudaSuccess ? CE_OK : CE_ERR_CUDA;
}

void ce_graph_destroy(ce_graph* g) {
  if (!g) return;
  cudaSetDevice(g->device);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
}

}  // extern "C"

// ---- autotuner ------------------------------------------------------------

namespace {

// Time one call on the engine's stream (after one untimed warm-up call).
template <typename F>
int time_call(ce_engine* e, F&& call, double* ms_out) {
  cudaEvent_t a, b;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return CE_ERR_CUDA;
  int rc = call();
  if (rc == CE_OK) {
    cudaEventRecord(a, e->stream);
    rc = call();
    cudaEventRecord(b, e->stream);
    if (rc == CE_OK && cudaEventSynchronize(b) != cudaSuccess) rc = CE_ERR_CUDA;
    float ms = 0.0f;
    if (rc == CE_OK) cudaEventElapsedTime(&ms, a, b);
    *ms_out = ms;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

struct Outputs {
  void* mem = nullptr;
  ce_outputs o{};
};

int alloc_outputs(ce_engine* e, uint64_t S, int atoms_per_row, Outputs* out) {
  const size_t mom = S * atoms_per_row * 3 * sizeof(float);
  const size_t total = mom + S * (sizeof(double) + sizeof(uint32_t) + 1) + 1024;
  cudaError_t st = cudaMalloc(&out->mem, total);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaMalloc(autotune outputs)");
  char* p = static_cast<char*>(out->mem);
  out->o.momenta = reinterpret_cast<float*>(p);
  p += (mom + 255) & ~static_cast<size_t>(255);
  out->o.ker = reinterpret_cast<double*>(p);
  p += ((S * sizeof(double)) + 255) & ~static_cast<size_t>(255);
  out->o.steps = reinterpret_cast<uint32_t*>(p);
  p += ((S * sizeof(uint32_t)) + 255) & ~static_cast<size_t>(255);
  out->o.status = reinterpret_cast<uint8_t*>(p);
  return CE_OK;
}

void record(ce_tune_result* report, int cap, int* n, const ce_tuning& t, double rate, int schedule) {
  if (report && *n < cap) {
    report[*n].t = t;
    report[*n].sims_per_s = rate;
    report[*n].schedule = schedule;
  }
  ++*n;
}

}  // namespace

extern "C" {

int ce_autotune_fixed(ce_engine* e, uint64_t S, const float* pos_dev, const ce_run_config* cfg,
                      ce_tune_result* report, int cap, int* n_report) {
  if (!e || !pos_dev || !cfg || S == 0) return CE_ERR_INVALID;
  if (!e->has_mol) return ce::fail(e, CE_ERR_STATE, "ce_autotune_fixed: no molecule set");
  if (cudaSetDevice(e->device) != cudaSuccess) return CE_ERR_CUDA;
  Outputs out;
  int rc = alloc_outputs(e, S, e->n, &out);
  if (rc != CE_OK) return rc;
  const ce_tuning saved = e->tuning;
  e->tuned_fixed[e->n].valid = false;
  // Layouts: one thread per sim, two threads per sim (3+ atoms), one lane per atom.
  std::vector<int> layouts = {1};
  if (e->n >= 3) layouts.push_back(2);
  if (e->n >= 2) layouts.push_back(e->n);
  const std::vector<int> blocks_atom = {64, 96, ce::kAtomMaxBlock};
  const int refills[] = {0, 1, 2, 4, 8};  // 0: the per-size default
  double best = -1.0;
  ce_tuning best_t{};
  int count = 0;
  for (int L : layouts)
    for (int B : (ce::layout_of(e->n, L) == ce::kLayoutAtom
                      ? blocks_atom  // the other two kernels fix their block size
                      : std::vector<int>{ce::fixed_launch_shape(e->n, ce::layout_of(e->n, L), cfg->precision_mode, 0).block}))
      for (int R : refills) {
        ce_tuning t{B, 0, R, L};
        e->tuning = t;
        double ms = 0.0;
        rc = time_call(e, [&] { return ce_run_device(e, S, pos_dev, cfg, &out.o, e->stream); }, &ms);
        if (rc != CE_OK) break;
        const double rate = ms > 0.0 ? static_cast<double>(S) / (ms * 1e-3) : 0.0;
        record(report, cap, &count, t, rate, CE_SCHEDULE_ONE_LAUNCH);
        if (rate > best) {
          best = rate;
          best_t = t;
        }
      }
  e->tuning = saved;
  cudaFree(out.mem);
  if (rc != CE_OK) return rc;
  e->tuned_fixed[e->n].valid = true;
  e->tuned_fixed[e->n].t = best_t;
  if (n_report) *n_report = std::min(count, cap);
  return CE_OK;
}

int ce_autotune_mixed(ce_engine* e, uint64_t S, const ce_mixed_batch* dev_in, double coulomb_k,
                      const ce_run_config* cfg, ce_tune_result* report, int cap, int* n_report, int* best_schedule) {
  if (!e || !dev_in || !cfg || S == 0) return CE_ERR_INVALID;
  if (cudaSetDevice(e->device) != cudaSuccess) return CE_ERR_CUDA;
  int rc = ce_reserve_mixed(e, S);
  if (rc != CE_OK) return rc;
  Outputs out;
  rc = alloc_outputs(e, S, CE_MAX_ATOMS, &out);
  if (rc != CE_OK) return rc;
  const ce_tuning saved = e->tuning;
  e->tuned_mixed.valid = false;
  const int blocks[] = {64, 96, ce::kAtomMaxBlock};
  const int refills[] = {0, 1, 2, 4};  // 0: each size's default
  const int schedules[] = {CE_SCHEDULE_ONE_LAUNCH, CE_SCHEDULE_PER_SIZE, CE_SCHEDULE_OVERLAP};
  double best = -1.0;
  ce_tuning best_t{};
  int best_s = CE_SCHEDULE_ONE_LAUNCH;
  int count = 0;
  // One lane per atom in every schedule and block size; two threads per sim
  // (lanes 2: 3+ atoms; its buckets fix their block, the 2-atom bucket keeps
  // 128 threads) in the two per-size schedules.
  for (int L : {0, 2})
    for (int sch : schedules)
      for (int B : blocks)
        for (int R : refills) {
        if (L == 2 && (sch == CE_SCHEDULE_ONE_LAUNCH || B != ce::kAtomMaxBlock)) continue;
        ce_tuning t{B, 0, R, L};
        e->tuning = t;
        double ms = 0.0;
        rc = time_call(e, [&] { return ce_run_mixed_device(e, S, dev_in, coulomb_k, cfg, &out.o, sch, e->stream); },
                       &ms);
        if (rc != CE_OK) break;
        const double rate = ms > 0.0 ? static_cast<double>(S) / (ms * 1e-3) : 0.0;
        record(report, cap, &count, t, rate, sch);
        if (rate > best) {
          best = rate;
          best_t = t;
          best_s = sch;
        }
      }
  e->tuning = saved;
  cudaFree(out.mem);
  if (rc != CE_OK) return rc;
  e->tuned_mixed.valid = true;
  e->tuned_mixed.t = best_t;
  e->tuned_schedule = best_s;
  if (best_schedule) *best_schedule = best_s;
  if (n_report) *n_report = std::min(count, cap);
  return CE_OK;
}

}  // extern "C"
