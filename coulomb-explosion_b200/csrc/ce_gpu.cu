// ce_gpu.cu -- C ABI of the B200 Coulomb-explosion engine (include/ce_gpu.h):
// engine lifetime, the fixed-molecule path and the host-buffer convenience path.
//
// Host side of the drop-in boundary: molecule constants (BatchedRK45 ctor,
// include/coulomb/batched_integrator.hpp:71-106), argument checks (the reference
// throws std::invalid_argument; here CE_ERR_INVALID) and the persistent launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>

#include "ce_gpu.h"
#include "engine.hpp"

namespace {

// Launch shape for one run: explicit tuning fields win, then the autotuned
// entry for this atom count, then the defaults (128 threads, occupancy-limited
// grid, the layout of default_lanes for this precision mode, the per-size refill
// granularity of default_refill).
ce_tuning effective_tuning(const ce_engine* e, int n, int mode) {
  ce_tuning t = e->tuning;
  const ce_tuned_entry& a = e->tuned_fixed[n];
  if (t.block_threads == 0) t.block_threads = a.valid && a.t.block_threads ? a.t.block_threads : 128;
  if (t.blocks_per_sm == 0 && a.valid) t.blocks_per_sm = a.t.blocks_per_sm;
  if (t.refill_threshold == 0 && a.valid) t.refill_threshold = a.t.refill_threshold;
  if (t.lanes_per_sim == 0)
    t.lanes_per_sim = a.valid && a.t.lanes_per_sim ? a.t.lanes_per_sim : ce::default_lanes(n, mode);
  if (n < 2) t.lanes_per_sim = 1;
  if (t.refill_threshold == 0) t.refill_threshold = ce::default_refill(n, t.lanes_per_sim);
  return t;
}

}  // namespace

extern "C" {

const char* ce_version(void) { return "ce_gpu 0.2 (sm_100a)"; }

void ce_default_config(ce_run_config* cfg) {
  if (!cfg) return;
  cfg->rtol = 1e-8;
  cfg->atol = 1e-16;
  cfg->pe_stop_fraction = 1e-9;
  cfg->max_dt = 1e12;
  cfg->max_steps = 1000000ull;
  cfg->redistribute_energy = 1;
  cfg->precision_mode = CE_PREC_FP32;
}

int ce_create(ce_engine** out, int device) {
  if (!out) return CE_ERR_INVALID;
  *out = nullptr;
  int count = 0;
  cudaError_t st = cudaGetDeviceCount(&count);
  if (st != cudaSuccess || count <= 0) return CE_ERR_NO_DEVICE;
  if (device < 0 || device >= count) return CE_ERR_INVALID;
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return CE_ERR_CUDA;
  if (prop.major < 10) return CE_ERR_NO_DEVICE;  // built for sm_100a only
  if (cudaSetDevice(device) != cudaSuccess) return CE_ERR_CUDA;
  ce_engine* e = new ce_engine();
  e->device = device;
  e->sms = prop.multiProcessorCount;
  if ((st = cudaMalloc(&e->d_cursor, sizeof(unsigned long long))) != cudaSuccess) {
    delete e;
    return CE_ERR_CUDA;
  }
  if ((st = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    cudaFree(e->d_cursor);
    delete e;
    return CE_ERR_CUDA;
  }
  *out = e;
  return CE_OK;
}

void ce_destroy(ce_engine* e) {
  if (!e) return;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  for (cudaStream_t x : {e->s_in, e->s_out, e->s_comp2, e->s_mix2})
    if (x) {
      cudaStreamSynchronize(x);
      cudaStreamDestroy(x);
    }
  for (int i = 0; i < 2; ++i)
    for (cudaEvent_t ev : {e->ev_loaded[i], e->ev_computed[i], e->ev_copied[i]})
      if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : {e->ev_mix_fork, e->ev_mix_join})
    if (ev) cudaEventDestroy(ev);
  if (e->d_arena) cudaFree(e->d_arena);
  if (e->h_io) cudaFreeHost(e->h_io);
  if (e->d_mixed) cudaFree(e->d_mixed);
  if (e->d_cursor) cudaFree(e->d_cursor);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

const char* ce_last_error(const ce_engine* e) { return e ? e->err.c_str() : "null engine"; }

int ce_last_launch_count(const ce_engine* e) { return e ? e->last_launches : 0; }

int ce_set_molecule(ce_engine* e, int n, const double* mass_me, const double* charge,
                    double coulomb_k) {
  if (!e) return CE_ERR_INVALID;
  if (n < 1 || n > CE_MAX_ATOMS)
    return ce::fail(e, CE_ERR_INVALID, "ce_set_molecule: n must be in 1..10");
  if (!mass_me || !charge) return ce::fail(e, CE_ERR_INVALID, "ce_set_molecule: NULL mass or charge");
  if (!std::isfinite(coulomb_k)) return ce::fail(e, CE_ERR_INVALID, "ce_set_molecule: non-finite k");
  ce::FixedMol m{};
  for (int i = 0; i < n; ++i) {
    if (!(mass_me[i] > 0.0) || !std::isfinite(mass_me[i]))
      return ce::fail(e, CE_ERR_INVALID, "ce_set_molecule: masses must be finite and > 0");
    if (!std::isfinite(charge[i]))
      return ce::fail(e, CE_ERR_INVALID, "ce_set_molecule: charges must be finite");
    m.mass[i] = mass_me[i];
    m.inv_m[i] = static_cast<float>(1.0 / mass_me[i]);
    m.q[i] = static_cast<float>(charge[i]);
    m.kq[i] = static_cast<float>(coulomb_k * charge[i]);
    m.k = static_cast<float>(coulomb_k);
    for (int j = 0; j < n; ++j)
      m.pc[i * n + j] = static_cast<float>(coulomb_k * charge[i] * charge[j]);
  }
  e->mol = m;
  e->n = n;
  e->has_mol = true;
  return CE_OK;
}

int ce_set_tuning(ce_engine* e, const ce_tuning* t) {
  if (!e || !t) return CE_ERR_INVALID;
  const ce_tuning v = *t;
  if (v.block_threads != 0 && (v.block_threads < 32 || v.block_threads > 256 || (v.block_threads % 32) != 0))
    return ce::fail(e, CE_ERR_INVALID, "ce_set_tuning: block_threads must be 0 or a multiple of 32 in 32..256");
  if (v.blocks_per_sm < 0 || v.blocks_per_sm > 64)
    return ce::fail(e, CE_ERR_INVALID, "ce_set_tuning: blocks_per_sm must be in 0..64");
  if (v.refill_threshold < 0 || v.refill_threshold > 32)
    return ce::fail(e, CE_ERR_INVALID, "ce_set_tuning: refill_threshold must be in 0..32");
  if (v.lanes_per_sim < 0 || v.lanes_per_sim > CE_MAX_ATOMS)
    return ce::fail(e, CE_ERR_INVALID,
                    "ce_set_tuning: lanes_per_sim must be 0 (auto), 1 (thread per sim), 2 (two threads per sim) or "
                    "3..10 (lane per atom)");
  e->tuning = v;
  return CE_OK;
}

int ce_get_tuning(const ce_engine* e, ce_tuning* t) {
  if (!e || !t) return CE_ERR_INVALID;
  *t = e->has_mol ? effective_tuning(e, e->n, 0) : e->tuning;
  return CE_OK;
}

}  // extern "C"

namespace ce {

int ensure_pipeline(ce_engine* e) {
  if (e->s_in) return CE_OK;
  cudaError_t st;
  if ((st = cudaStreamCreateWithFlags(&e->s_in, cudaStreamNonBlocking)) != cudaSuccess ||
      (st = cudaStreamCreateWithFlags(&e->s_out, cudaStreamNonBlocking)) != cudaSuccess ||
      (st = cudaStreamCreateWithFlags(&e->s_comp2, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_fail(e, st, "cudaStreamCreate(pipeline streams)");
  for (int i = 0; i < 2; ++i)
    if ((st = cudaEventCreateWithFlags(&e->ev_loaded[i], cudaEventDisableTiming)) != cudaSuccess ||
        (st = cudaEventCreateWithFlags(&e->ev_computed[i], cudaEventDisableTiming)) != cudaSuccess ||
        (st = cudaEventCreateWithFlags(&e->ev_copied[i], cudaEventDisableTiming)) != cudaSuccess)
      return cuda_fail(e, st, "cudaEventCreate");
  return CE_OK;
}

}  // namespace ce

namespace {

// Launch shape of a fixed-molecule run: kernel, block, dynamic shared memory,
// resident blocks per SM and simulations per block.
struct FixedShape {
  ce::FixedKernelFn fn = nullptr;
  int block = 0;
  size_t smem = 0;
  int per_sm = 0;
  uint64_t sims_per_block = 0;
  int refill = 0;
  int layout = 0;
};

int fixed_shape(ce_engine* e, int mode, FixedShape* sh) {
  cudaError_t st;
  const ce_tuning t = effective_tuning(e, e->n, mode);
  ce_engine::FixedShapeCache& c = e->shape_cache;
  if (c.valid && c.n == e->n && c.mode == mode && c.t.block_threads == t.block_threads &&
      c.t.blocks_per_sm == t.blocks_per_sm && c.t.refill_threshold == t.refill_threshold &&
      c.t.lanes_per_sim == t.lanes_per_sim) {
    sh->fn = c.fn;
    sh->block = c.block;
    sh->smem = c.smem;
    sh->per_sm = c.per_sm;
    sh->sims_per_block = c.sims_per_block;
    sh->refill = t.refill_threshold;
    sh->layout = c.layout;
    return CE_OK;
  }
  c.valid = false;
  const int layout = ce::layout_of(e->n, t.lanes_per_sim);
  sh->fn = layout == ce::kLayoutAtom   ? ce::select_atom_kernel(e->n, mode)
           : layout == ce::kLayoutPair ? ce::select_pair_kernel(e->n, mode)
                                       : ce::select_fixed_kernel(e->n, mode);
  if (!sh->fn) return ce::fail(e, CE_ERR_INVALID, "ce_run: no kernel for this atom count");
  // The thread-per-sim and two-thread kernels fix their block size at compile
  // time (their shared-memory offsets are immediates) and keep their stage
  // accelerations in dynamic shared memory.
  const ce::FixedLaunchShape ls = ce::fixed_launch_shape(e->n, layout, mode, t.block_threads);
  sh->block = ls.block;
  sh->sims_per_block = ls.sims_per_block;
  sh->refill = t.refill_threshold;
  sh->smem = ls.smem;
  sh->layout = layout;
  if (sh->smem > 0) {
    st = cudaFuncSetAttribute(reinterpret_cast<const void*>(sh->fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                              static_cast<int>(sh->smem));
    if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaFuncSetAttribute(max dynamic shared memory)");
    // All of the SM's unified L1 / shared storage as shared memory: the kernel
    // reads almost nothing through L1, and CH4's seven stage slots per thread
    // need 56 KB per block for four blocks per SM.
    st = cudaFuncSetAttribute(reinterpret_cast<const void*>(sh->fn), cudaFuncAttributePreferredSharedMemoryCarveout,
                              cudaSharedmemCarveoutMaxShared);
    if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaFuncSetAttribute(shared memory carveout)");
  }
  sh->per_sm = t.blocks_per_sm;
  if (sh->per_sm == 0) {
    st = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sh->per_sm, sh->fn, sh->block, sh->smem);
    if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (sh->per_sm < 1) sh->per_sm = 1;
  }
  c.n = e->n;
  c.mode = mode;
  c.t = t;
  c.fn = sh->fn;
  c.block = sh->block;
  c.smem = sh->smem;
  c.per_sm = sh->per_sm;
  c.sims_per_block = sh->sims_per_block;
  c.layout = sh->layout;
  c.valid = true;
  return CE_OK;
}

// One fixed-molecule launch on `s`, its work queue at `cursor` (reset to 0 on
// `s` first). Arguments are checked by the callers.
int launch_fixed(ce_engine* e, uint64_t S, const float* pos, const ce_run_config* cfg, const ce_outputs* out,
                 cudaStream_t s, unsigned long long* cursor) {
  FixedShape sh;
  int rc = fixed_shape(e, cfg->precision_mode, &sh);
  if (rc != CE_OK) return rc;
  const ce::FixedKernelFn fn = sh.fn;
  const int block = sh.block;
  const size_t smem = sh.smem;
  const int per_sm = sh.per_sm;
  const uint64_t sims_per_block = sh.sims_per_block;
  const uint64_t need_blocks = (S + sims_per_block - 1) / sims_per_block;
  const uint64_t grid = std::min<uint64_t>(static_cast<uint64_t>(e->sms) * per_sm, need_blocks);

  ce::RunParams P{};
  ce::fill_run_params(P, cfg, out, sh.refill);
  P.pos = pos;
  P.cursor = cursor;
  P.S = S;

  cudaError_t st = cudaMemsetAsync(cursor, 0, sizeof(unsigned long long), s);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaMemsetAsync(cursor)");
  fn<<<static_cast<unsigned>(grid), block, smem, s>>>(P, e->mol);
  st = cudaGetLastError();
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "rk45 kernel launch");
  e->last_launches = 1;
  return CE_OK;
}

// Streamed host-buffer run (the thread-per-sim and two-thread layouts): ONE
// persistent launch over all S sims in device buffers, with the copies around
// it. Positions go up in kIoMaxChunks-bounded chunks on the copy-in stream,
// each followed by a 4-byte copy that marks the chunk present (io_ready); the
// kernel's warps wait (bounded) for the chunk of the sims they claim. Every
// finished sim is counted toward its chunk, and the count that completes a
// chunk raises a flag in mapped host memory; the host, polling those flags in
// order, sends each chunk's results down on the copy-out stream while the
// kernel goes on. Nothing between the first chunk's upload and the last
// chunk's download waits on a chunk boundary: no per-chunk kernel tails, no
// slot reuse. Every wait the host makes is bounded and a failure raises the
// abort word, which ends the kernel's input waits.
using ce::kIoMinChunk;
// run_streamed's result when the kernel's input waits ran out (no other error).
constexpr int kIoWaitRanOut = 1000;

// Whether the GPU's work may be serialised for this process: blocking launches,
// or a tool injected into the CUDA runtime (profilers and checkers serialise
// kernels and copies). The streamed run needs its copies to run beside its
// kernel, so ce_run then uses the chunked pipeline.
bool gpu_work_serialised() {
  const char* blocking = std::getenv("CUDA_LAUNCH_BLOCKING");
  if (blocking && std::strcmp(blocking, "0") != 0) return true;
  const char* injected = std::getenv("CUDA_INJECTION64_PATH");
  return injected && injected[0] != '\0';
}
constexpr size_t kIoHeader = 4096;  // cursor, error, ready flags, done counters
constexpr size_t kIoMaxArena = 8ull << 30;

size_t al256(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }

// Device bytes of a streamed run of S sims with the outputs `out` asks for.
size_t streamed_bytes(const ce_engine* e, uint64_t S, const ce_outputs* out) {
  const size_t n3 = static_cast<size_t>(e->n) * 3;
  size_t b = kIoHeader + 2 * al256(S * n3 * sizeof(float));  // positions in, momenta out
  if (out->positions) b += al256(S * n3 * sizeof(float));
  for (const void* p : {static_cast<const void*>(out->ker), static_cast<const void*>(out->t_final),
                        static_cast<const void*>(out->pe_final), static_cast<const void*>(out->ke_before),
                        static_cast<const void*>(out->e0)})
    if (p) b += al256(S * sizeof(double));
  if (out->steps) b += al256(S * sizeof(uint32_t));
  if (out->rejects) b += al256(S * sizeof(uint32_t));
  if (out->status) b += al256(S);
  return b;
}

int run_streamed(ce_engine* e, uint64_t S, const float* pos, const ce_run_config* cfg, const ce_outputs* out,
                 const FixedShape& sh) {
  cudaError_t st;
  const size_t n3 = static_cast<size_t>(e->n) * 3;
  const size_t total = streamed_bytes(e, S, out);
  if (total > e->arena_bytes) {
    cudaDeviceSynchronize();
    if (e->d_arena) cudaFree(e->d_arena);
    e->d_arena = nullptr;
    e->arena_bytes = 0;
    st = cudaMalloc(&e->d_arena, total);
    if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaMalloc(arena)");
    e->arena_bytes = total;
  }
  if (!e->h_io) {
    st = cudaHostAlloc(reinterpret_cast<void**>(&e->h_io), ce::kIoWords * sizeof(unsigned), cudaHostAllocMapped);
    if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaHostAlloc(io flags)");
    st = cudaHostGetDevicePointer(reinterpret_cast<void**>(&e->h_io_dev), e->h_io, 0);
    if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaHostGetDevicePointer(io flags)");
  }
  const unsigned io_shift = ce::io_chunk_shift(S);
  const uint64_t io_chunk = 1ull << io_shift;
  const uint64_t J = (S + io_chunk - 1) / io_chunk;

  char* base = static_cast<char*>(e->d_arena);
  auto* cursor = reinterpret_cast<unsigned long long*>(base);
  auto* ready = reinterpret_cast<unsigned*>(base + 256);
  auto* done = reinterpret_cast<unsigned long long*>(base + 1024);
  char* b = base + kIoHeader;
  auto take = [&](size_t bytes) {
    char* r = b;
    b += al256(bytes);
    return r;
  };
  auto* d_pos = reinterpret_cast<float*>(take(S * n3 * sizeof(float)));
  ce_outputs d{};
  d.momenta = reinterpret_cast<float*>(take(S * n3 * sizeof(float)));
  if (out->positions) d.positions = reinterpret_cast<float*>(take(S * n3 * sizeof(float)));
  if (out->ker) d.ker = reinterpret_cast<double*>(take(S * sizeof(double)));
  if (out->t_final) d.t_final = reinterpret_cast<double*>(take(S * sizeof(double)));
  if (out->pe_final) d.pe_final = reinterpret_cast<double*>(take(S * sizeof(double)));
  if (out->ke_before) d.ke_before = reinterpret_cast<double*>(take(S * sizeof(double)));
  if (out->e0) d.e0 = reinterpret_cast<double*>(take(S * sizeof(double)));
  if (out->steps) d.steps = reinterpret_cast<uint32_t*>(take(S * sizeof(uint32_t)));
  if (out->rejects) d.rejects = reinterpret_cast<uint32_t*>(take(S * sizeof(uint32_t)));
  if (out->status) d.status = reinterpret_cast<uint8_t*>(take(S));

  volatile unsigned* hio = e->h_io;
  for (int k = 0; k < ce::kIoWords; ++k) hio[k] = 0u;
  hio[ce::kIoOne] = 1u;

  const ce::FixedKernelFn fn = ce::select_io_kernel(e->n, cfg->precision_mode, sh.layout == ce::kLayoutPair);
  if (!fn) return ce::fail(e, CE_ERR_INVALID, "ce_run: no streamed kernel for this atom count");
  if (sh.smem > 0) {  // the same attributes as the plain kernel of this layout
    st = cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                              static_cast<int>(sh.smem));
    if (st == cudaSuccess)
      st = cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared);
    if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaFuncSetAttribute(streamed kernel)");
  }
  ce::RunParams P{};
  ce::fill_run_params(P, cfg, &d, sh.refill);
  P.pos = d_pos;
  P.cursor = cursor;
  P.S = S;
  P.io_ready = ready;
  P.io_done = done;
  P.io_host_done = e->h_io_dev;
  P.io_abort = e->h_io_dev + ce::kIoAbort;
  P.io_error = e->h_io_dev + ce::kIoError;
  P.io_shift = io_shift;
  const uint64_t need_blocks = (S + sh.sims_per_block - 1) / sh.sims_per_block;
  const uint64_t grid = std::min<uint64_t>(static_cast<uint64_t>(e->sms) * sh.per_sm, need_blocks);

  // header zeroed, then the kernel; the uploads start once the header is zero
  st = cudaMemsetAsync(base, 0, kIoHeader, e->stream);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaMemsetAsync(io header)");
  int rc = ce::record(e, e->ev_loaded[0], e->stream);
  if (rc != CE_OK) return rc;
  fn<<<static_cast<unsigned>(grid), sh.block, sh.smem, e->stream>>>(P, e->mol);
  st = cudaGetLastError();
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "rk45 streamed kernel launch");
  e->last_launches = 1;

  // From here on the kernel may be waiting for input: any failure raises the
  // abort word before returning.
  auto abort_run = [&](int code) {
    hio[ce::kIoAbort] = 1u;
    cudaStreamSynchronize(e->stream);
    cudaStreamSynchronize(e->s_in);
    cudaStreamSynchronize(e->s_out);
    return code;
  };
  if ((rc = ce::wait_on(e, e->s_in, e->ev_loaded[0])) != CE_OK) return abort_run(rc);
  for (uint64_t j = 0; j < J; ++j) {
    const uint64_t s0 = j * io_chunk, Sj = std::min<uint64_t>(S, s0 + io_chunk) - s0;
    st = cudaMemcpyAsync(d_pos + s0 * n3, pos + s0 * n3, Sj * n3 * sizeof(float), cudaMemcpyHostToDevice, e->s_in);
    if (st == cudaSuccess)
      st = cudaMemcpyAsync(ready + j, e->h_io + ce::kIoOne, sizeof(unsigned), cudaMemcpyHostToDevice, e->s_in);
    if (st != cudaSuccess) return abort_run(ce::cuda_fail(e, st, "cudaMemcpyAsync(streamed H2D)"));
  }
  if ((rc = ce::record(e, e->ev_loaded[1], e->s_in)) != CE_OK) return abort_run(rc);
  // Results down, chunk by chunk as the kernel completes them. The host waits
  // at most kIoHostWaitSeconds for one chunk, and stops waiting once the kernel
  // has ended without completing it. If the input copies have not all landed
  // within a few seconds of the launch (far longer than they take beside the
  // kernel), the copies are being held back until the kernel ends (a tool that
  // serialises GPU work, not caught by gpu_work_serialised): the host raises the
  // abort word, the kernel's waits end at their next check, and ce_run falls
  // back to the chunked pipeline instead of waiting for the waits to run out.
  constexpr double kIoHostWaitSeconds = 120.0;
  const double input_deadline = 2.0 + static_cast<double>(S * n3 * sizeof(float)) * 1e-9;  // >= 1 GB/s
  const auto t_launch = std::chrono::steady_clock::now();
  bool inputs_landed = false;
  for (uint64_t j = 0; j < J; ++j) {
    const auto t0 = std::chrono::steady_clock::now();
    for (uint64_t spin = 1; hio[j] == 0u; ++spin) {
      if ((spin & 1023u) == 0u) {
        const cudaError_t q = cudaStreamQuery(e->stream);
        if (q != cudaErrorNotReady && hio[j] == 0u) {
          if (q != cudaSuccess) return abort_run(ce::cuda_fail(e, q, "streamed kernel"));
          return abort_run(ce::fail(e, CE_ERR_CUDA, "ce_run: the streamed kernel ended before finishing a chunk"));
        }
        const auto now = std::chrono::steady_clock::now();
        if (!inputs_landed && std::chrono::duration<double>(now - t_launch).count() > input_deadline) {
          const cudaError_t qi = cudaEventQuery(e->ev_loaded[1]);
          if (qi == cudaErrorNotReady) {
            abort_run(CE_OK);
            return kIoWaitRanOut;
          }
          if (qi != cudaSuccess) return abort_run(ce::cuda_fail(e, qi, "streamed input copies"));
          inputs_landed = true;
        }
        if (std::chrono::duration<double>(now - t0).count() > kIoHostWaitSeconds)
          return abort_run(ce::fail(e, CE_ERR_CUDA, "ce_run: timed out waiting for a streamed chunk"));
        std::this_thread::yield();
      }
    }
    const uint64_t s0 = j * io_chunk, Sj = std::min<uint64_t>(S, s0 + io_chunk) - s0;
    struct Copy {
      void* dst;
      const void* src;
      size_t bytes;
    } copies[] = {
        {out->momenta + s0 * n3, d.momenta + s0 * n3, Sj * n3 * sizeof(float)},
        {out->ker ? out->ker + s0 : nullptr, d.ker + s0, Sj * sizeof(double)},
        {out->t_final ? out->t_final + s0 : nullptr, d.t_final + s0, Sj * sizeof(double)},
        {out->pe_final ? out->pe_final + s0 : nullptr, d.pe_final + s0, Sj * sizeof(double)},
        {out->ke_before ? out->ke_before + s0 : nullptr, d.ke_before + s0, Sj * sizeof(double)},
        {out->e0 ? out->e0 + s0 : nullptr, d.e0 + s0, Sj * sizeof(double)},
        {out->steps ? out->steps + s0 : nullptr, d.steps + s0, Sj * sizeof(uint32_t)},
        {out->rejects ? out->rejects + s0 : nullptr, d.rejects + s0, Sj * sizeof(uint32_t)},
        {out->status ? out->status + s0 : nullptr, d.status + s0, Sj},
        {out->positions ? out->positions + s0 * n3 : nullptr, d.positions + s0 * n3, Sj * n3 * sizeof(float)}};
    for (const Copy& c : copies) {
      if (!c.dst) continue;
      st = cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, e->s_out);
      if (st != cudaSuccess) return abort_run(ce::cuda_fail(e, st, "cudaMemcpyAsync(streamed D2H)"));
    }
  }
  st = cudaStreamSynchronize(e->s_out);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e->stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e->s_in);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaStreamSynchronize");
  if (hio[ce::kIoError] != 0u) return kIoWaitRanOut;
  return CE_OK;
}

}  // namespace

extern "C" {

int ce_run_device(ce_engine* e, uint64_t S, const float* pos, const ce_run_config* cfg,
                  const ce_outputs* out, void* stream) {
  if (!e) return CE_ERR_INVALID;
  e->last_launches = 0;
  int rc = ce::check_config(e, cfg);
  if (rc != CE_OK) return rc;
  if (!e->has_mol) return ce::fail(e, CE_ERR_STATE, "ce_run: no molecule set (ce_set_molecule)");
  if (S == 0) return CE_OK;
  if (!pos || !out || !out->momenta)
    return ce::fail(e, CE_ERR_INVALID, "ce_run: pos and out->momenta are required");
  if (S > (1ull << 40)) return ce::fail(e, CE_ERR_INVALID, "ce_run: S too large");
  const cudaError_t st = cudaSetDevice(e->device);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaSetDevice");
  return launch_fixed(e, S, pos, cfg, out, static_cast<cudaStream_t>(stream), e->d_cursor);
}

// Host-buffer path, pipelined: the batch is cut into chunks that alternate
// between two device slots; chunk k's positions go up on a copy-in stream while
// chunk k-1 integrates and chunk k-2's results come down on a copy-out stream.
// With pinned host buffers the copies overlap the kernels. The two slots
// integrate on two compute streams with a work-queue cursor each, so a chunk's
// persistent blocks take over SMs as the previous chunk's blocks retire instead
// of waiting for its last simulation.
constexpr uint64_t kResidentQuartersPerChunk = 8;  // 2x the resident sims

int ce_run(ce_engine* e, uint64_t S, const float* pos, const ce_run_config* cfg,
           const ce_outputs* out) {
  if (!e) return CE_ERR_INVALID;
  int rc = ce::check_config(e, cfg);
  if (rc != CE_OK) return rc;
  if (!e->has_mol) return ce::fail(e, CE_ERR_STATE, "ce_run: no molecule set (ce_set_molecule)");
  if (S == 0) return CE_OK;
  if (!pos || !out || !out->momenta)
    return ce::fail(e, CE_ERR_INVALID, "ce_run: pos and out->momenta are required");
  if (S > (1ull << 40)) return ce::fail(e, CE_ERR_INVALID, "ce_run: S too large");
  cudaError_t st = cudaSetDevice(e->device);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaSetDevice");
  rc = ce::ensure_pipeline(e);
  if (rc != CE_OK) return rc;

  // Chunking: up to 16 chunks, each at least kResidentQuartersPerChunk / 4
  // times the sims the persistent grid holds at once (and 2^16), so a chunk's
  // last simulations are a small part of its run. One chunk below twice that.
  // Measured on CH4 1e6 with the thread-per-sim kernel (75,776 sims resident),
  // end to end: 1x the resident count 2.29e8/s, 1.5x 2.37e8, 2x 2.40-2.47e8,
  // 2.5x 2.27e8, 3x 2.25e8, 4x 2.19e8 (device-resident 2.74-2.78e8); with a
  // fixed 2^16 minimum 2.24e8.
  FixedShape sh;
  rc = fixed_shape(e, cfg->precision_mode, &sh);
  if (rc != CE_OK) return rc;
  // The thread-per-sim and two-thread layouts stream their I/O around one
  // launch (run_streamed) when the whole batch fits the device arena bound.
  // If its input waits run out (the copies did not run beside the kernel), the
  // call is redone by the chunked pipeline and the engine stops streaming.
  if (sh.layout != ce::kLayoutAtom && S >= 2 * kIoMinChunk && S < (1ull << 31) && !e->streamed_off &&
      !gpu_work_serialised() && streamed_bytes(e, S, out) <= kIoMaxArena) {
    rc = run_streamed(e, S, pos, cfg, out, sh);
    if (rc != kIoWaitRanOut) return rc;
    e->streamed_off = true;
  }
  const uint64_t resident = static_cast<uint64_t>(e->sms) * static_cast<uint64_t>(sh.per_sm) * sh.sims_per_block;
  const uint64_t min_chunk = std::max<uint64_t>(1ull << 16, kResidentQuartersPerChunk * resident / 4);
  uint64_t bnd[17], C = 0;
  const uint64_t nchunks = ce::chunk_bounds(S, min_chunk, 16, bnd, &C);
  auto bound = [&](uint64_t k) -> uint64_t { return bnd[k]; };
  const size_t n3 = static_cast<size_t>(e->n) * 3;
  auto al = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
  const size_t b_pos = al(C * n3 * sizeof(float));
  const size_t b_d = al(C * sizeof(double));
  const size_t b_u = al(C * sizeof(uint32_t));
  const size_t b_s = al(C);
  const size_t slot_bytes = 3 * b_pos + 5 * b_d + 2 * b_u + b_s;  // pos, momenta, positions out, ...
  const int nslots = nchunks > 1 ? 2 : 1;
  constexpr size_t kCursorBytes = 256;  // one work-queue cursor per slot
  const size_t total = kCursorBytes + slot_bytes * nslots;
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
    float* pos;
    ce_outputs d;
    unsigned long long* cursor;
    cudaStream_t s;
  } slots[2];
  for (int k = 0; k < nslots; ++k) {
    char* b = static_cast<char*>(e->d_arena) + kCursorBytes + k * slot_bytes;
    Slot& sl = slots[k];
    sl.cursor = static_cast<unsigned long long*>(e->d_arena) + k;
    sl.s = k == 0 ? e->stream : e->s_comp2;
    sl.pos = reinterpret_cast<float*>(b);
    b += b_pos;
    sl.d = ce_outputs{};
    sl.d.momenta = reinterpret_cast<float*>(b);
    b += b_pos;
    float* xo = reinterpret_cast<float*>(b);
    b += b_pos;
    double* dd[5];
    for (int i = 0; i < 5; ++i, b += b_d) dd[i] = reinterpret_cast<double*>(b);
    uint32_t* du[2];
    for (int i = 0; i < 2; ++i, b += b_u) du[i] = reinterpret_cast<uint32_t*>(b);
    sl.d.ker = out->ker ? dd[0] : nullptr;
    sl.d.t_final = out->t_final ? dd[1] : nullptr;
    sl.d.pe_final = out->pe_final ? dd[2] : nullptr;
    sl.d.ke_before = out->ke_before ? dd[3] : nullptr;
    sl.d.e0 = out->e0 ? dd[4] : nullptr;
    sl.d.positions = out->positions ? xo : nullptr;
    sl.d.steps = out->steps ? du[0] : nullptr;
    sl.d.rejects = out->rejects ? du[1] : nullptr;
    sl.d.status = out->status ? reinterpret_cast<uint8_t*>(b) : nullptr;
  }

  int launches = 0;
  for (uint64_t k = 0; k < nchunks; ++k) {
    const uint64_t s0 = bound(k);
    const uint64_t Sk = bound(k + 1) - s0;
    if (Sk == 0) continue;
    const int sl = static_cast<int>(k % nslots);
    Slot& slot = slots[sl];
    // positions up once the slot's previous chunk has been integrated
    if (k >= 2 && (rc = ce::wait_on(e, e->s_in, e->ev_computed[sl])) != CE_OK) return rc;
    st = cudaMemcpyAsync(slot.pos, pos + s0 * n3, Sk * n3 * sizeof(float), cudaMemcpyHostToDevice, e->s_in);
    if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaMemcpyAsync(pos H2D)");
    if ((rc = ce::record(e, e->ev_loaded[sl], e->s_in)) != CE_OK) return rc;
    // integrate once the positions are in and the slot's previous results are out
    if ((rc = ce::wait_on(e, slot.s, e->ev_loaded[sl])) != CE_OK) return rc;
    if (k >= 2 && (rc = ce::wait_on(e, slot.s, e->ev_copied[sl])) != CE_OK) return rc;
    rc = launch_fixed(e, Sk, slot.pos, cfg, &slot.d, slot.s, slot.cursor);
    if (rc != CE_OK) return rc;
    launches += e->last_launches;
    if ((rc = ce::record(e, e->ev_computed[sl], slot.s)) != CE_OK) return rc;
    // results down
    if ((rc = ce::wait_on(e, e->s_out, e->ev_computed[sl])) != CE_OK) return rc;
    struct Copy {
      void* dst;
      const void* src;
      size_t bytes;
    } copies[] = {
        {out->momenta ? out->momenta + s0 * n3 : nullptr, slot.d.momenta, Sk * n3 * sizeof(float)},
        {out->ker ? out->ker + s0 : nullptr, slot.d.ker, Sk * sizeof(double)},
        {out->t_final ? out->t_final + s0 : nullptr, slot.d.t_final, Sk * sizeof(double)},
        {out->pe_final ? out->pe_final + s0 : nullptr, slot.d.pe_final, Sk * sizeof(double)},
        {out->ke_before ? out->ke_before + s0 : nullptr, slot.d.ke_before, Sk * sizeof(double)},
        {out->steps ? out->steps + s0 : nullptr, slot.d.steps, Sk * sizeof(uint32_t)},
        {out->rejects ? out->rejects + s0 : nullptr, slot.d.rejects, Sk * sizeof(uint32_t)},
        {out->status ? out->status + s0 : nullptr, slot.d.status, Sk},
        {out->positions ? out->positions + s0 * n3 : nullptr, slot.d.positions, Sk * n3 * sizeof(float)},
        {out->e0 ? out->e0 + s0 : nullptr, slot.d.e0, Sk * sizeof(double)}};
    for (const Copy& c : copies) {
      if (!c.dst) continue;
      st = cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, e->s_out);
      if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaMemcpyAsync(D2H)");
    }
    if ((rc = ce::record(e, e->ev_copied[sl], e->s_out)) != CE_OK) return rc;
  }
  e->last_launches = launches;
  st = cudaStreamSynchronize(e->s_out);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e->stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e->s_comp2);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaStreamSynchronize");
  return CE_OK;
}

}  // extern "C"
