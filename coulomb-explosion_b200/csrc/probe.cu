// probe.cu -- FP32 FMA throughput probe and the bounded-wait check
// (include/ce_probe.h).
#include <cuda_runtime.h>

#include <algorithm>

#include "ce_gpu.h"
#include "ce_probe.h"
#include "umma.cuh"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 2048;
constexpr int kUnroll = 16;  // FMAs between loop-control instructions: 8 x 16

__global__ void __launch_bounds__(256) ffma_probe(float* out, float b, float c) {
  float a[kChains];
#pragma unroll
  for (int i = 0; i < kChains; ++i) a[i] = static_cast<float>(threadIdx.x + i);
  for (int it = 0; it < kIters; ++it) {
#pragma unroll
    for (int i = 0; i < kChains; ++i) a[i] = fmaf(a[i], b, c);
  }
  float s = 0.0f;
#pragma unroll
  for (int i = 0; i < kChains; ++i) s += a[i];
  if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

// Long-running variants: `iters` outer iterations of kUnroll x kChains
// independent FMAs per thread, scalar FFMA or packed FFMA2 (two FP32 FMAs per
// instruction, per-element IEEE rounding), so the kernel runs for tens of
// milliseconds and the clock settles under load.
__global__ void __launch_bounds__(256) ffma_probe_long(float* out, float b, float c, int iters) {
  float a[kChains];
#pragma unroll
  for (int i = 0; i < kChains; ++i) a[i] = static_cast<float>(threadIdx.x + i);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
      for (int i = 0; i < kChains; ++i) a[i] = fmaf(a[i], b, c);
    }
  }
  float s = 0.0f;
#pragma unroll
  for (int i = 0; i < kChains; ++i) s += a[i];
  if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) ffma2_probe_long(float* out, float b, float c, int iters) {
  float2 a[kChains];
  const float2 bb = make_float2(b, b), cc = make_float2(c, c);
#pragma unroll
  for (int i = 0; i < kChains; ++i)
    a[i] = make_float2(static_cast<float>(threadIdx.x + i), static_cast<float>(threadIdx.x + 2 * i));
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
      for (int i = 0; i < kChains; ++i) a[i] = __ffma2_rn(a[i], bb, cc);
    }
  }
  float s = 0.0f;
#pragma unroll
  for (int i = 0; i < kChains; ++i) s += a[i].x + a[i].y;
  if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// An mbarrier that nothing arrives on, waited for with the same bounded poll
// the tensor-core kernels use: the wait must give up, record its code and let
// the kernel finish.
__global__ void bounded_wait_probe(int* err, uint32_t spins) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) ce::umma::mbar_init(&bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) ce::umma::mbar_wait(&bar, 0u, err, 7, spins);
}

}  // namespace

extern "C" int ce_probe_bounded_wait(int device, unsigned spins, int* code_out) {
  if (!code_out || spins == 0 || spins > (1u << 20)) return CE_ERR_INVALID;
  *code_out = 0;
  if (cudaSetDevice(device) != cudaSuccess) return CE_ERR_NO_DEVICE;
  int* d = nullptr;
  if (cudaMalloc(&d, sizeof(int)) != cudaSuccess) return CE_ERR_CUDA;
  int rc = CE_OK;
  if (cudaMemset(d, 0, sizeof(int)) != cudaSuccess) rc = CE_ERR_CUDA;
  if (rc == CE_OK) {
    bounded_wait_probe<<<1, 32>>>(d, spins);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(code_out, d, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = CE_ERR_CUDA;
  }
  cudaFree(d);
  return rc;
}

extern "C" int ce_probe_fp32_peak(int device, double* tflops_out) {
  if (!tflops_out) return CE_ERR_INVALID;
  *tflops_out = 0.0;
  if (cudaSetDevice(device) != cudaSuccess) return CE_ERR_NO_DEVICE;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return CE_ERR_CUDA;
  const int block = 256, per_sm = 8;
  const int grid = sms * per_sm;
  float* out = nullptr;
  if (cudaMalloc(&out, sizeof(float) * grid * block) != cudaSuccess) return CE_ERR_CUDA;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best_ms = 1e30f;
  int rc = CE_OK;
  for (int rep = 0; rep < 6; ++rep) {
    cudaEventRecord(e0);
    ffma_probe<<<grid, block>>>(out, 0.999999f, 1e-7f);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      rc = CE_ERR_CUDA;
      break;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best_ms) best_ms = ms;  // rep 0 is warm-up
  }
  if (cudaGetLastError() != cudaSuccess) rc = CE_ERR_CUDA;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (rc != CE_OK) return rc;
  const double flops = 2.0 * kChains * static_cast<double>(kIters) * grid * block;
  *tflops_out = flops / (best_ms * 1e-3) / 1e12;
  return CE_OK;
}

extern "C" int ce_probe_fp32_peak_ex(int device, int packed, double min_ms, double* tflops_out, double* ms_out) {
  if (!tflops_out || min_ms < 0.0 || min_ms > 1000.0 || (packed != 0 && packed != 1)) return CE_ERR_INVALID;
  *tflops_out = 0.0;
  if (ms_out) *ms_out = 0.0;
  if (cudaSetDevice(device) != cudaSuccess) return CE_ERR_NO_DEVICE;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return CE_ERR_CUDA;
  const int block = 256, per_sm = 8;
  const int grid = sms * per_sm;
  float* out = nullptr;
  if (cudaMalloc(&out, sizeof(float) * grid * block) != cudaSuccess) return CE_ERR_CUDA;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int rc = CE_OK;
  auto launch = [&](int iters) {
    if (packed)
      ffma2_probe_long<<<grid, block>>>(out, 0.999999f, 1e-7f, iters);
    else
      ffma_probe_long<<<grid, block>>>(out, 0.999999f, 1e-7f, iters);
  };
  auto timed = [&](int iters, float* ms) {
    cudaEventRecord(e0);
    launch(iters);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess) return false;
    return cudaEventElapsedTime(ms, e0, e1) == cudaSuccess;
  };
  // size the run: grow the iteration count until one launch lasts min_ms
  int iters = 64;
  float ms = 0.0f;
  for (int k = 0; k < 20; ++k) {
    if (!timed(iters, &ms)) {
      rc = CE_ERR_CUDA;
      break;
    }
    if (ms >= min_ms || iters >= (1 << 24)) break;
    const double grow = ms > 0.0f ? (min_ms * 1.1) / ms : 16.0;
    iters = static_cast<int>(std::min<double>(1 << 24, std::max<double>(2.0 * iters, iters * grow)));
  }
  float best_ms = 1e30f;
  for (int rep = 0; rc == CE_OK && rep < 5; ++rep) {
    if (!timed(iters, &ms)) {
      rc = CE_ERR_CUDA;
      break;
    }
    best_ms = std::min(best_ms, ms);
  }
  if (cudaGetLastError() != cudaSuccess) rc = CE_ERR_CUDA;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (rc != CE_OK) return rc;
  const double fma_per_thread = static_cast<double>(iters) * kUnroll * kChains * (packed ? 2 : 1);
  *tflops_out = 2.0 * fma_per_thread * grid * block / (best_ms * 1e-3) / 1e12;
  if (ms_out) *ms_out = best_ms;
  return CE_OK;
}
