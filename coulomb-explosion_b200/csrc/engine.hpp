// engine.hpp -- the engine object behind the C ABI and the helpers the host
// translation units share (ce_gpu.cu: fixed molecule; mixed.cu: mixed batches,
// graphs, autotuning).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "ce_gpu.h"
#include "rk45_atom.cuh"
#include "rk45_sim.cuh"

struct ce_tuned_entry {
  bool valid = false;
  ce_tuning t{};
};

struct ce_engine {
  int device = 0;
  int sms = 0;
  bool has_mol = false;
  int n = 0;
  ce::FixedMol mol{};
  ce_tuning tuning{0, 0, 0, 0};  // all fields automatic (autotuned entry, else default)
  // Autotuned launch shapes, per atom count (fixed path) and for the mixed path.
  ce_tuned_entry tuned_fixed[CE_MAX_ATOMS + 1];
  ce_tuned_entry tuned_mixed;
  int tuned_schedule = CE_SCHEDULE_ONE_LAUNCH;  // schedule ce_run_mixed uses (autotuner's pick)
  unsigned long long* d_cursor = nullptr;  // fixed path work-queue head (engine scratch)
  cudaStream_t stream = nullptr;           // stream of the host-buffer paths
  // ce_run pipelining: copy-in / copy-out streams, a second compute stream (the
  // chunks of the two device slots integrate on `stream` and `s_comp2`, so one
  // chunk's blocks start while the other's last simulations finish) and per-slot
  // events
  cudaStream_t s_in = nullptr, s_out = nullptr, s_comp2 = nullptr;
  cudaEvent_t ev_loaded[2] = {nullptr, nullptr}, ev_computed[2] = {nullptr, nullptr},
              ev_copied[2] = {nullptr, nullptr};
  void* d_arena = nullptr;                 // device buffers of the host-buffer paths
  size_t arena_bytes = 0;
  // Mixed-batch scratch: 4 x 11 u64 bucket tables, then the S-entry permutation.
  void* d_mixed = nullptr;
  size_t mixed_bytes = 0;
  // CE_SCHEDULE_OVERLAP: a side stream and its fork / join events
  cudaStream_t s_mix2 = nullptr;
  cudaEvent_t ev_mix_fork = nullptr, ev_mix_join = nullptr;
  int last_launches = 0;
  // Launch shape of the last fixed-molecule run (ce_gpu.cu fixed_shape), reused
  // while the atom count, precision mode and effective tuning are unchanged, so
  // the chunks of a ce_run set kernel attributes and query occupancy once.
  struct FixedShapeCache {
    bool valid = false;
    int n = 0, mode = 0;
    ce_tuning t{};
    ce::FixedKernelFn fn = nullptr;
    int block = 0;
    size_t smem = 0;
    int per_sm = 0;
    unsigned long long sims_per_block = 0;
    int layout = 0;
  } shape_cache;
  // Streamed ce_run (ce_gpu.cu run_streamed): mapped pinned host words, words
  // [0, kIoMaxChunks) the per-chunk done flags the kernel raises, then the abort
  // word the host raises, the constant 1 the input-ready copies read, and the
  // kernel's error word copied back.
  unsigned* h_io = nullptr;
  unsigned* h_io_dev = nullptr;
  // Set once a streamed run's input waits ran out (the copies it waits for did
  // not run beside the kernel: a tool that serialises the GPU's work); ce_run
  // then uses the chunked pipeline.
  bool streamed_off = false;
  std::string err;
};

namespace ce {
constexpr int kIoMaxChunks = 64;
constexpr uint64_t kIoMinChunk = 16384;
// Chunk size of a streamed ce_run of S sims, as a power of two 2^shift (the
// kernel shifts instead of dividing): at least kIoMinChunk sims, fewer than
// kIoMaxChunks / 2 chunks. A chunk of 2^shift sims is a whole number of 128-byte
// lines of positions for any atom count, so no cache line spans two chunks.
inline unsigned io_chunk_shift(uint64_t S) {
  unsigned shift = 0;
  while ((1ull << shift) < kIoMinChunk || (S >> shift) >= static_cast<uint64_t>(kIoMaxChunks / 2)) ++shift;
  return shift;
}
constexpr int kIoAbort = kIoMaxChunks, kIoOne = kIoMaxChunks + 1, kIoError = kIoMaxChunks + 2;
constexpr int kIoWords = kIoMaxChunks + 4;
}  // namespace ce

namespace ce {

inline int fail(ce_engine* e, int code, const std::string& msg) {
  if (e) e->err = msg;
  return code;
}

inline int cuda_fail(ce_engine* e, cudaError_t st, const char* what) {
  return fail(e, CE_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(st));
}

inline int check_config(ce_engine* e, const ce_run_config* cfg) {
  if (!cfg) return fail(e, CE_ERR_INVALID, "ce_run: cfg is NULL");
  if (!(cfg->rtol >= 0.0) || !(cfg->atol >= 0.0) || !std::isfinite(cfg->rtol) || !std::isfinite(cfg->atol))
    return fail(e, CE_ERR_INVALID, "ce_run: rtol and atol must be finite and >= 0");
  if (!(cfg->rtol > 0.0 || cfg->atol > 0.0))
    return fail(e, CE_ERR_INVALID, "ce_run: rtol and atol cannot both be 0");
  if (!(cfg->max_dt > 0.0)) return fail(e, CE_ERR_INVALID, "ce_run: max_dt must be > 0");
  if (!std::isfinite(cfg->pe_stop_fraction))
    return fail(e, CE_ERR_INVALID, "ce_run: pe_stop_fraction must be finite");
  if (cfg->precision_mode < 0 || cfg->precision_mode > 3)
    return fail(e, CE_ERR_INVALID, "ce_run: precision_mode must be a combination of CE_PREC_* bits");
  return CE_OK;
}

inline void fill_run_params(RunParams& P, const ce_run_config* cfg, const ce_outputs* out, int refill_threshold) {
  P.momenta = out->momenta;
  P.ker = out->ker;
  P.steps = out->steps;
  P.status = out->status;
  P.rejects = out->rejects;
  P.t_final = out->t_final;
  P.pe_final = out->pe_final;
  P.ke_before = out->ke_before;
  P.positions = out->positions;
  P.e0 = out->e0;
  P.rtol = static_cast<float>(cfg->rtol);
  P.atol = static_cast<float>(cfg->atol);
  P.max_dt = static_cast<float>(cfg->max_dt);
  P.pe_stop_f = static_cast<float>(cfg->pe_stop_fraction);
  P.pe_stop_d = cfg->pe_stop_fraction;
  P.max_steps = cfg->max_steps > 0xffffffffull ? 0xffffffffu : static_cast<uint32_t>(cfg->max_steps);
  P.redistribute = cfg->redistribute_energy ? 1 : 0;
  P.refill_threshold = refill_threshold;
}

inline FixedKernelFn select_fixed_kernel(int n, int mode) {
  switch (mode & 3) {
    case 0: return fixed_kernel_m0(n);
    case 1: return fixed_kernel_m1(n);
    case 2: return fixed_kernel_m2(n);
    default: return fixed_kernel_m3(n);
  }
}

inline FixedKernelFn select_pair_kernel(int n, int mode) {
  switch (mode & 3) {
    case 0: return pair_kernel_m0(n);
    case 1: return pair_kernel_m1(n);
    case 2: return pair_kernel_m2(n);
    default: return pair_kernel_m3(n);
  }
}

inline FixedKernelFn select_io_kernel(int n, int mode, bool pair) {
  switch (mode & 3) {
    case 0: return io_kernel_m0(n, pair);
    case 1: return io_kernel_m1(n, pair);
    case 2: return io_kernel_m2(n, pair);
    default: return io_kernel_m3(n, pair);
  }
}

inline PairBucketFn select_pair_bucket_kernel(int n, int mode) {
  switch (mode & 3) {
    case 0: return pair_bucket_kernel_m0(n);
    case 1: return pair_bucket_kernel_m1(n);
    case 2: return pair_bucket_kernel_m2(n);
    default: return pair_bucket_kernel_m3(n);
  }
}

inline AtomKernelFn select_atom_kernel(int n, int mode) {
  switch (mode & 3) {
    case 0: return atom_kernel_m0(n);
    case 1: return atom_kernel_m1(n);
    case 2: return atom_kernel_m2(n);
    default: return atom_kernel_m3(n);
  }
}

inline MixedKernelFn select_mixed_kernel(int n, int mode) {
  switch (mode & 3) {
    case 0: return mixed_kernel_m0(n);
    case 1: return mixed_kernel_m1(n);
    case 2: return mixed_kernel_m2(n);
    default: return mixed_kernel_m3(n);
  }
}

// ce_run_mixed_device_state with one extra switch: skip_empty leaves rows with
// n_atoms == 0 untouched instead of writing CE_SIM_BAD_INPUT outputs (the
// closure's plain continuation of the sims its gate sent back). Defined in mixed.cu.
int run_mixed_device(ce_engine* e, uint64_t S, const ce_mixed_batch* in, double coulomb_k, const ce_run_config* cfg,
                     const ce_outputs* out, int schedule, void* stream, bool skip_empty, const ce_sim_state* resume,
                     const ce_sim_state* save);


// Chunk bounds of the pipelined host-buffer paths: nchunks = 1 below
// 2 * min_chunk sims, else min(max_chunks, S / min_chunk) (max_chunks <= 16); chunk
// k spans [bnd[k], bnd[k + 1]). From 6 chunks on, the first and last two are
// tapered (weights 1/4, 1/2, 1, ..., 1, 1/2, 1/4), which keeps the copy-in before
// the first kernel and the copy-out after the last short. Returns nchunks; *cmax is
// the largest chunk.
inline uint64_t chunk_bounds(uint64_t S, uint64_t min_chunk, uint64_t max_chunks, uint64_t (&bnd)[17],
                             uint64_t* cmax) {
  const uint64_t nchunks = S < 2 * min_chunk ? 1 : (S / min_chunk < max_chunks ? S / min_chunk : max_chunks);
  const bool taper = nchunks >= 6;
  auto w = [&](uint64_t k) -> uint64_t {  // in quarters
    if (!taper) return 4;
    if (k == 0 || k + 1 == nchunks) return 1;
    if (k == 1 || k + 2 == nchunks) return 2;
    return 4;
  };
  uint64_t wsum = 0;
  for (uint64_t k = 0; k < nchunks; ++k) wsum += w(k);
  uint64_t acc = 0;
  for (uint64_t k = 0; k < nchunks; ++k) {
    bnd[k] = S * acc / wsum;  // S <= 2^40 and acc <= 64: no overflow
    acc += w(k);
  }
  bnd[nchunks] = S;
  uint64_t c = 0;
  for (uint64_t k = 0; k < nchunks; ++k) c = bnd[k + 1] - bnd[k] > c ? bnd[k + 1] - bnd[k] : c;
  *cmax = c;
  return nchunks;
}

// Event record / stream wait of the pipelined host-buffer paths, checked: a
// dependency that failed to register would let a copy race its kernel.
inline int record(ce_engine* e, cudaEvent_t ev, cudaStream_t s) {
  const cudaError_t st = cudaEventRecord(ev, s);
  return st == cudaSuccess ? CE_OK : cuda_fail(e, st, "cudaEventRecord");
}
inline int wait_on(ce_engine* e, cudaStream_t s, cudaEvent_t ev) {
  const cudaError_t st = cudaStreamWaitEvent(s, ev, 0);
  return st == cudaSuccess ? CE_OK : cuda_fail(e, st, "cudaStreamWaitEvent");
}

// Creates, once per engine, the copy-in / copy-out streams, the second compute
// stream and the per-slot events of the pipelined host-buffer paths. Defined in
// ce_gpu.cu.
int ensure_pipeline(ce_engine* e);

}  // namespace ce
