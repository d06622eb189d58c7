// noalloc.cu -- ce_run_device_noalloc: the fixed-molecule integration for
// callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: code that runs inside a framework which
// owns every device allocation (a pooled allocator, a memory-budgeted serving
// process, an embedding host with a fixed arena), or callers that set up once
// and must not touch the allocator afterwards. They still own their input and
// output buffers; what they cannot provide is the kernel's own scratch, here
// the persistent kernel's work-queue cursor. This entry point keeps that
// scratch in a file-scope device array instead, and calls no cudaMalloc,
// cudaFree or allocating library routine.
//
// Scratch: kNoallocScratchWords 64-bit words (256 bytes) of static device
// memory, held by every GPU that loads this library until the process exits.
// The kernel uses one word (the cursor); the need does not grow with the
// number of simulations, and requests outside the supported sizes (n outside
// 1..10, S above 2^40) are rejected before anything is launched.
//
// Host code never passes the array's name to a kernel: on the host that name is
// only a stand-in, not a device address. The first call on each device, with
// that device current, looks the address up once with cudaGetSymbolAddress and
// caches it; that first call should therefore come before any stream capture.
// The cached address is valid for the life of the device's primary context: a
// cudaDeviceReset between calls is not supported (the module reloads and the
// array can move).
// Every call shares the one cursor and leaves its last value behind, so each
// call clears it (cudaMemsetAsync on the caller's stream) before the launch;
// calls whose launches overlap on the GPU (different streams, no ordering)
// race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "ce_gpu.h"
#include "rk45_atom.cuh"
#include "rk45_sim.cuh"

namespace {

constexpr int kNoallocScratchWords = 32;  // 256 bytes
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoallocScratchWords];

std::mutex g_setup_mu;
unsigned long long* g_scratch_addr[kMaxDevices] = {};

int report(char* err, size_t err_len, int code, const char* msg) {
  if (err && err_len > 0) std::snprintf(err, err_len, "%s", msg);
  return code;
}

// Once per device (the caller's current device): resolve the array's device
// address. Returns CE_OK and sets *addr, or an error code.
int scratch_address(int dev, unsigned long long** addr, char* err, size_t err_len) {
  if (dev < 0 || dev >= kMaxDevices)
    return report(err, err_len, CE_ERR_INVALID, "ce_run_device_noalloc: device index out of range");
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t st = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (st != cudaSuccess || !p) {
      char msg[256];
      std::snprintf(msg, sizeof msg, "ce_run_device_noalloc: cudaGetSymbolAddress failed: %s",
                    cudaGetErrorString(st));
      return report(err, err_len, CE_ERR_CUDA, msg);
    }
    g_scratch_addr[dev] = static_cast<unsigned long long*>(p);
  }
  *addr = g_scratch_addr[dev];
  return CE_OK;
}

// The kernel ce_run_device launches by default (ce::default_lanes): one thread
// per simulation, two threads per simulation, or one lane per atom.
ce::FixedKernelFn kernel_for(int n, int mode) {
  const int layout = ce::layout_of(n, ce::default_lanes(n, mode));
  if (layout == ce::kLayoutAtom) {
    switch (mode & 3) {
      case 0: return ce::atom_kernel_m0(n);
      case 1: return ce::atom_kernel_m1(n);
      case 2: return ce::atom_kernel_m2(n);
      default: return ce::atom_kernel_m3(n);
    }
  }
  if (layout == ce::kLayoutPair) {
    switch (mode & 3) {
      case 0: return ce::pair_kernel_m0(n);
      case 1: return ce::pair_kernel_m1(n);
      case 2: return ce::pair_kernel_m2(n);
      default: return ce::pair_kernel_m3(n);
    }
  }
  switch (mode & 3) {
    case 0: return ce::fixed_kernel_m0(n);
    case 1: return ce::fixed_kernel_m1(n);
    case 2: return ce::fixed_kernel_m2(n);
    default: return ce::fixed_kernel_m3(n);
  }
}

}  // namespace

extern "C" int ce_run_device_noalloc(int n, const double* mass_me, const double* charge,
                                     double coulomb_k, uint64_t S, const float* pos,
                                     const ce_run_config* cfg, const ce_outputs* out, void* stream,
                                     char* err, size_t err_len) {
  if (n < 1 || n > CE_MAX_ATOMS)
    return report(err, err_len, CE_ERR_INVALID, "ce_run_device_noalloc: n must be in 1..10 atoms");
  if (S > (1ull << 40))
    return report(err, err_len, CE_ERR_INVALID, "ce_run_device_noalloc: S above the 2^40 maximum");
  if (!mass_me || !charge || !cfg)
    return report(err, err_len, CE_ERR_INVALID, "ce_run_device_noalloc: NULL mass, charge or cfg");
  if (!std::isfinite(coulomb_k))
    return report(err, err_len, CE_ERR_INVALID, "ce_run_device_noalloc: non-finite Coulomb constant");
  if (!(cfg->rtol >= 0.0) || !(cfg->atol >= 0.0) || !std::isfinite(cfg->rtol) ||
      !std::isfinite(cfg->atol) || !(cfg->rtol > 0.0 || cfg->atol > 0.0) || !(cfg->max_dt > 0.0) ||
      !std::isfinite(cfg->pe_stop_fraction) || cfg->precision_mode < 0 || cfg->precision_mode > 3)
    return report(err, err_len, CE_ERR_INVALID, "ce_run_device_noalloc: invalid run configuration");
  ce::FixedMol m{};
  for (int i = 0; i < n; ++i) {
    if (!(mass_me[i] > 0.0) || !std::isfinite(mass_me[i]) || !std::isfinite(charge[i]))
      return report(err, err_len, CE_ERR_INVALID,
                    "ce_run_device_noalloc: masses must be finite and > 0, charges finite");
    m.mass[i] = mass_me[i];
    m.inv_m[i] = static_cast<float>(1.0 / mass_me[i]);
    m.q[i] = static_cast<float>(charge[i]);
    m.kq[i] = static_cast<float>(coulomb_k * charge[i]);
    for (int j = 0; j < n; ++j) m.pc[i * n + j] = static_cast<float>(coulomb_k * charge[i] * charge[j]);
  }
  m.k = static_cast<float>(coulomb_k);
  if (S == 0) return CE_OK;
  if (!pos || !out || !out->momenta)
    return report(err, err_len, CE_ERR_INVALID, "ce_run_device_noalloc: pos and out->momenta are required");

  int dev = 0;
  cudaError_t st = cudaGetDevice(&dev);
  if (st != cudaSuccess) return report(err, err_len, CE_ERR_CUDA, "ce_run_device_noalloc: cudaGetDevice failed");
  unsigned long long* cursor = nullptr;
  int rc = scratch_address(dev, &cursor, err, err_len);
  if (rc != CE_OK) return rc;

  const ce::FixedKernelFn fn = kernel_for(n, cfg->precision_mode);
  const int lanes = ce::default_lanes(n, cfg->precision_mode);
  // The thread-per-sim and two-thread kernels take their stage slots as dynamic
  // shared memory (on-chip, per block; not an allocation).
  const ce::FixedLaunchShape ls =
      ce::fixed_launch_shape(n, ce::layout_of(n, lanes), cfg->precision_mode, ce::kAtomMaxBlock);
  const int block = ls.block;
  const size_t smem = ls.smem;
  if (smem > 0 &&
      (cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                            static_cast<int>(smem)) != cudaSuccess ||
       cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributePreferredSharedMemoryCarveout,
                            cudaSharedmemCarveoutMaxShared) != cudaSuccess))
    return report(err, err_len, CE_ERR_CUDA, "ce_run_device_noalloc: shared-memory attribute failed");
  int per_sm = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, smem) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return report(err, err_len, CE_ERR_CUDA, "ce_run_device_noalloc: device query failed");
  if (per_sm < 1) per_sm = 1;
  const uint64_t sims_per_block = ls.sims_per_block;
  const uint64_t need = (S + sims_per_block - 1) / sims_per_block;
  const uint64_t grid = need < static_cast<uint64_t>(sms) * per_sm ? need : static_cast<uint64_t>(sms) * per_sm;

  ce::RunParams P{};
  P.pos = pos;
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
  P.cursor = cursor;
  P.S = S;
  P.rtol = static_cast<float>(cfg->rtol);
  P.atol = static_cast<float>(cfg->atol);
  P.max_dt = static_cast<float>(cfg->max_dt);
  P.pe_stop_f = static_cast<float>(cfg->pe_stop_fraction);
  P.pe_stop_d = cfg->pe_stop_fraction;
  P.max_steps = cfg->max_steps > 0xffffffffull ? 0xffffffffu : static_cast<uint32_t>(cfg->max_steps);
  P.redistribute = cfg->redistribute_energy ? 1 : 0;
  P.refill_threshold = ce::default_refill(n, lanes);

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  st = cudaMemsetAsync(cursor, 0, sizeof(unsigned long long), s);  // the cursor must start at 0
  if (st != cudaSuccess) return report(err, err_len, CE_ERR_CUDA, "ce_run_device_noalloc: clearing the cursor failed");
  fn<<<static_cast<unsigned>(grid), block, smem, s>>>(P, m);
  st = cudaGetLastError();
  if (st != cudaSuccess) {
    char msg[256];
    std::snprintf(msg, sizeof msg, "ce_run_device_noalloc: launch failed: %s", cudaGetErrorString(st));
    return report(err, err_len, CE_ERR_CUDA, msg);
  }
  return CE_OK;
}
