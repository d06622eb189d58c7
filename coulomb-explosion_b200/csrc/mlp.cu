// mlp.cu -- the closure network: a BF16 MLP (FP32 accumulation) trained and
// served by hand-written sm_100a kernels (include/ce_closure.h).
//
// Every product (forward, input gradient, weight gradient) runs through one
// tcgen05 GEMM kernel: a CTA owns a 128-row tile and up to 256 columns, stages
// 64-wide K slices of both operands into shared memory in the canonical
// no-swizzle layout (either operand K-major or MN-major, so transposes cost
// nothing), issues four 128xNx16 tcgen05.mma per slice from one thread with the
// accumulator in tensor memory, and runs a fused epilogue (bias + SiLU, bias
// only in FP32, SiLU' gating, or FP32 atomics for split-K weight gradients).
// Small elementwise kernels cover the loss, bias gradients and Adam.
//
// No counterpart in the reference (its pipeline has no learned component).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "ce_closure.h"
#include "ce_gpu.h"
#include "umma.cuh"

namespace ce {
namespace mlp {

using bf16 = __nv_bfloat16;

enum Epi : int {
  kEpiFwdAct = 0,        // Z = acc + b (bf16), Y = silu(Z) (bf16)
  kEpiFwdLinearF32 = 1,  // C = acc + b (f32)
  kEpiBwdAct = 2,        // Y = acc * silu'(Z) (bf16)
  kEpiStoreBf16 = 3,     // Y = acc (bf16)
  kEpiAtomicF32 = 4,     // C[m][n] += acc
  kEpiAtomicF32T = 5,    // C[n][m] += acc
};

struct GemmArgs {
  const bf16* A;
  int lda;
  const bf16* B;
  int ldb;
  int M, N, K;
  int k_split;
  int epi;
  const float* bias;
  bf16* Y;
  int ldy;
  const bf16* Zin;
  bf16* Zout;
  int ldz;
  float* C;
  int ldc;
  int* err;
};

constexpr int kTM = 128;      // UMMA M
constexpr int kKC = 64;       // K elements staged per slice
constexpr int kTNmax = 256;   // UMMA N (columns per CTA)
constexpr int kLBO = 128;     // bytes between K-adjacent core matrices
constexpr int kSBO = (kKC / 8) * 128;  // bytes between M/N-adjacent core matrices
constexpr int kSmemA = kTM * kKC * 2;      // 16 KB
constexpr int kSmemB = kTNmax * kKC * 2;   // 32 KB
constexpr int kSmemBytes = kSmemA + kSmemB + 64;
constexpr uint32_t kTmemCols = 256;

// Stage rows [r0, r0 + R) x K slice [k0, k0 + kKC) of a logical operand
// Op(r, k) into canonical layout. MN_MAJOR: memory holds G[k][r] (r
// contiguous); otherwise G[r][k]. Out-of-range elements are zero.
template <bool MN_MAJOR>
__device__ __forceinline__ void stage(uint8_t* s, const bf16* G, int ld, int r0, int rmax, int k0, int kend, int R) {
  const int chunks = R * (kKC / 8);
  for (int t = threadIdx.x; t < chunks; t += blockDim.x) {
    int r, kk;
    uint4 v = make_uint4(0, 0, 0, 0);
    uint32_t off;
    if (!MN_MAJOR) {
      r = t / (kKC / 8);
      const int kc = t % (kKC / 8);
      kk = kc * 8;
      if (r0 + r < rmax && k0 + kk < kend) v = *reinterpret_cast<const uint4*>(G + static_cast<size_t>(r0 + r) * ld + k0 + kk);
      off = (r / 8) * kSBO + kc * kLBO + (r % 8) * 16;
    } else {
      kk = t / (R / 8);
      const int mc = t % (R / 8);
      r = mc * 8;
      if (r0 + r < rmax && k0 + kk < kend) v = *reinterpret_cast<const uint4*>(G + static_cast<size_t>(k0 + kk) * ld + r0 + r);
      off = mc * kSBO + (kk / 8) * kLBO + (kk % 8) * 16;
    }
    *reinterpret_cast<uint4*>(s + off) = v;
  }
}

// sigmoid(z) = (1 + tanh(z/2)) / 2 with the hardware tanh approximation
// (tanh.approx.f32, max relative error ~2^-11, below the BF16 rounding of the
// activations): one special-function op per element instead of exp + divide.
__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sigmoidf_(float z) { return fmaf(0.5f, tanh_approx(0.5f * z), 0.5f); }

// Forward SiLU of a BF16 pre-activation in BF16 arithmetic:
// y = z * (1/2 + tanh(z/2)/2) (tanh.approx.bf16). The fused serving kernel
// evaluates the same operations on pairs (bf16x2), so both forwards agree bit
// for bit.
__device__ __forceinline__ bf16 silu_bf16(bf16 z) {
  const bf16 half = __float2bfloat16(0.5f);
  const bf16 h = __hmul(z, half);
  uint16_t tb;
  asm("tanh.approx.bf16 %0, %1;" : "=h"(tb) : "h"(__bfloat16_as_ushort(h)));
  return __hmul(z, __hfma(__ushort_as_bfloat16(tb), half, half));
}

template <bool A_MN, bool B_MN>
__global__ void __launch_bounds__(128) umma_gemm_kernel(const GemmArgs g) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sA = smem;
  uint8_t* sB = smem + kSmemA;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kSmemA + kSmemB);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kSmemA + kSmemB + 16);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kTM;
  const int n0 = blockIdx.y * kTNmax;
  const int TN = min(kTNmax, g.N - n0);
  const int kbeg = blockIdx.z * g.k_split;
  const int kend = min(g.K, kbeg + g.k_split);
  if (tid == 0) umma::mbar_init(bar, 1);
  if (warp == 0) umma::tmem_alloc(tslot, kTmemCols);
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = umma::instr_desc_bf16_f32(kTM, TN, A_MN, B_MN);
  uint32_t phase = 0;
  bool ok = true;
  for (int k0 = kbeg; k0 < kend && ok; k0 += kKC) {
    stage<A_MN>(sA, g.A, g.lda, m0, g.M, k0, kend, kTM);
    stage<B_MN>(sB, g.B, g.ldb, n0, g.N, k0, kend, TN);
    umma::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      umma::tc_fence_after();
      const uint32_t a0 = umma::smem_addr(sA), b0 = umma::smem_addr(sB);
#pragma unroll
      for (int ks = 0; ks < kKC / 16; ++ks) {
        const uint64_t ad = umma::smem_desc(a0 + ks * 2 * kLBO, kLBO, kSBO);
        const uint64_t bd = umma::smem_desc(b0 + ks * 2 * kLBO, kLBO, kSBO);
        umma::mma_bf16(tmem, ad, bd, idesc, (k0 > kbeg || ks > 0) ? 1u : 0u);
      }
      umma::mma_commit(bar);
    }
    const bool w = umma::mbar_wait(bar, phase, g.err, 1);
    phase ^= 1u;
    ok = __syncthreads_and(w) != 0;  // also orders the next slice's smem writes after the MMAs
  }
  umma::tc_fence_after();
  if (ok) {
    const int row = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < TN; c0 += 16) {
      uint32_t r[16];
      umma::tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0), r);
      umma::tmem_wait_ld();
      if (row >= g.M) continue;
      const int nb = n0 + c0;
      if (nb + 16 <= g.N && g.epi != kEpiAtomicF32T && g.epi != kEpiFwdLinearF32) {
        // full 16-column chunk: vector stores (16 B of BF16 / float4 atomics)
        if (g.epi == kEpiAtomicF32) {
          float4* c = reinterpret_cast<float4*>(g.C + static_cast<size_t>(row) * g.ldc + nb);
#pragma unroll
          for (int q = 0; q < 4; ++q)
            atomicAdd(c + q, make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]),
                                         __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3])));
          continue;
        }
        uint32_t y[8], z[8];
        if (g.epi == kEpiBwdAct) {
          const uint4* zi = reinterpret_cast<const uint4*>(g.Zin + static_cast<size_t>(row) * g.ldz + nb);
          const uint4 z0 = zi[0], z1 = zi[1];
          const uint32_t zw[8] = {z0.x, z0.y, z0.z, z0.w, z1.x, z1.y, z1.z, z1.w};
#pragma unroll
          for (int q = 0; q < 8; ++q) z[q] = zw[q];
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          bf16 o0, o1;
          const float a0 = __uint_as_float(r[2 * q]), a1 = __uint_as_float(r[2 * q + 1]);
          if (g.epi == kEpiFwdAct) {
            const bf16 z0 = __float2bfloat16(a0 + g.bias[nb + 2 * q]);
            const bf16 z1 = __float2bfloat16(a1 + g.bias[nb + 2 * q + 1]);
            z[q] = static_cast<uint32_t>(__bfloat16_as_ushort(z0)) | (static_cast<uint32_t>(__bfloat16_as_ushort(z1)) << 16);
            o0 = silu_bf16(z0);
            o1 = silu_bf16(z1);
          } else if (g.epi == kEpiBwdAct) {
            const float za = __bfloat162float(__ushort_as_bfloat16(static_cast<unsigned short>(z[q] & 0xffffu)));
            const float zb = __bfloat162float(__ushort_as_bfloat16(static_cast<unsigned short>(z[q] >> 16)));
            const float sa = sigmoidf_(za), sb = sigmoidf_(zb);
            o0 = __float2bfloat16(a0 * (sa * (1.0f + za * (1.0f - sa))));
            o1 = __float2bfloat16(a1 * (sb * (1.0f + zb * (1.0f - sb))));
          } else {
            o0 = __float2bfloat16(a0);
            o1 = __float2bfloat16(a1);
          }
          y[q] = static_cast<uint32_t>(__bfloat16_as_ushort(o0)) | (static_cast<uint32_t>(__bfloat16_as_ushort(o1)) << 16);
        }
        uint4* yo = reinterpret_cast<uint4*>(g.Y + static_cast<size_t>(row) * g.ldy + nb);
        yo[0] = make_uint4(y[0], y[1], y[2], y[3]);
        yo[1] = make_uint4(y[4], y[5], y[6], y[7]);
        if (g.epi == kEpiFwdAct) {
          uint4* zo = reinterpret_cast<uint4*>(g.Zout + static_cast<size_t>(row) * g.ldz + nb);
          zo[0] = make_uint4(z[0], z[1], z[2], z[3]);
          zo[1] = make_uint4(z[4], z[5], z[6], z[7]);
        }
        continue;
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int n = n0 + c0 + j;
        if (n >= g.N) break;
        const float acc = __uint_as_float(r[j]);
        switch (g.epi) {
          case kEpiFwdAct: {
            const bf16 zb = __float2bfloat16(acc + g.bias[n]);
            g.Zout[static_cast<size_t>(row) * g.ldz + n] = zb;
            g.Y[static_cast<size_t>(row) * g.ldy + n] = silu_bf16(zb);
            break;
          }
          case kEpiFwdLinearF32:
            g.C[static_cast<size_t>(row) * g.ldc + n] = acc + g.bias[n];
            break;
          case kEpiBwdAct: {
            const float z = __bfloat162float(g.Zin[static_cast<size_t>(row) * g.ldz + n]);
            const float s = sigmoidf_(z);
            g.Y[static_cast<size_t>(row) * g.ldy + n] = __float2bfloat16(acc * (s * (1.0f + z * (1.0f - s))));
            break;
          }
          case kEpiStoreBf16:
            g.Y[static_cast<size_t>(row) * g.ldy + n] = __float2bfloat16(acc);
            break;
          case kEpiAtomicF32:
            atomicAdd(g.C + static_cast<size_t>(row) * g.ldc + n, acc);
            break;
          default:
            atomicAdd(g.C + static_cast<size_t>(n) * g.ldc + row, acc);
            break;
        }
      }
    }
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, kTmemCols);
}

// ---- elementwise kernels ----

// dOut = 2 (out - t) w / sum(w); loss += sum (out - t)^2 w / sum(w).
__global__ void mse_grad_kernel(const float* out, const float* t, const float* w, float inv_wsum, int n_total,
                                bf16* dout, float* loss) {
  float acc = 0.0f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_total; i += gridDim.x * blockDim.x) {
    const float d = (out[i] - t[i]) * w[i];
    dout[i] = __float2bfloat16(2.0f * d * inv_wsum);
    acc += d * (out[i] - t[i]) * inv_wsum;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc);
}

// db[n] += sum_rows dZ[row][n]; blockIdx.y takes a slice of kColRows rows, so
// the rows are summed in parallel (one atomic per column and slice).
constexpr int kColRows = 256;
__global__ void colsum_kernel(const bf16* dz, int rows, int cols, int ld, float* db) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= cols) return;
  const int r0 = blockIdx.y * kColRows, r1 = min(rows, r0 + kColRows);
  float s = 0.0f;
#pragma unroll 8
  for (int r = r0; r < r1; ++r) s += __bfloat162float(dz[static_cast<size_t>(r) * ld + n]);
  atomicAdd(db + n, s);
}

// Adam (Kingma & Ba 2015) on FP32 master weights; refreshes the BF16 copy.
__global__ void adam_kernel(float* p, const float* g, float* m, float* v, bf16* pb, int n, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float upd = lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] -= upd;
    if (pb) pb[i] = __float2bfloat16(p[i]);
  }
}

__global__ void f32_to_bf16_kernel(const float* a, bf16* b, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = __float2bfloat16(a[i]);
}

// ---- fused forward (serving) ----
//
// One persistent CTA per SM walks pairs of 128-row tiles through every layer,
// with warp roles:
//   warp 0  producer: one thread streams the weights, pre-packed in global
//           memory in the tensor core's canonical operand layout (one
//           contiguous block per 64-wide K slice), into a three-slot ring with
//           1-D bulk copies (cp.async.bulk, completion counted on an mbarrier);
//   warp 1  MMA issuer: one thread runs the (layer, tile) jobs in the order
//           A0 B0 A1 B1 ..., each job's slices into its tile's accumulator
//           (two 128 x 256 FP32 blocks, 512 TMEM columns);
//   warps 2-13 / 14-25  epilogue of tile A / tile B (12 warps a tile: each of
//           the 4 TMEM lane quarters by 3 warps, one third of the columns each,
//           so that enough warps hide the TMEM-load and SiLU latencies): TMEM -> bias + SiLU ->
//           BF16 -> the tile's activation operand in shared memory (the input
//           of the next layer), or FP32 outputs after the last layer; they also
//           load the next input tile.
// So tile A's epilogue of layer l overlaps tile B's MMAs of layer l and vice
// versa; activations never leave shared memory. All waits are bounded.
constexpr int kFwdMaxLayers = 8;
constexpr int kFwdGroups = 3;                  // epilogue column groups per tile
constexpr int kFwdThreads = 32 * (2 + 2 * 4 * kFwdGroups);  // producer, MMA issuer, 2 x 12 epilogue
constexpr int kFwdKmax = 256;                  // widest layer input held in shared memory
constexpr int kFwdSboA = (kFwdKmax / 8) * 128; // 4096 B between row-adjacent core matrices
constexpr int kFwdAct = kTM * kFwdKmax * 2;    // 64 KB activation operand per tile
constexpr int kFwdW = kTNmax * kKC * 2;        // 32 KB per weight slice slot
constexpr int kFwdSlots = 3;
constexpr int kFwdSmem = 2 * kFwdAct + kFwdSlots * kFwdW + 256;
constexpr uint32_t kFwdTmemCols = 512;

struct FwdArgs {
  const bf16* x;     // [rows][fan_in[0]]
  const uint8_t* wpk;  // packed weight slices
  const float* p;    // FP32 parameters (biases)
  float* out;        // [rows][fan_out[L-1]]
  int rows;
  int layers;
  int fan_in[kFwdMaxLayers], fan_out[kFwdMaxLayers], b_off[kFwdMaxLayers], w_off[kFwdMaxLayers];
  int slice_off[kFwdMaxLayers][4];  // byte offset of slice (l, c) in wpk; slice size = fan_out * 128 B
  int* err;
};

__device__ __forceinline__ void cp_async16(void* s, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(umma::smem_addr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(umma::smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(umma::smem_addr(bar)), "r"(bytes)
               : "memory");
}
// 1-D bulk copy global -> this CTA's shared memory, completion reported as
// transaction bytes on `bar`; the destination is this CTA alone.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   umma::smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(umma::smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ uint32_t tanh_bf16x2(uint32_t x) {
  uint32_t y;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(y) : "r"(x));
  return y;
}

// SiLU of two pre-activations, rounded like the training forward: z = BF16(acc
// + b), then y = z * (1/2 + tanh(z/2)/2) in BF16x2 arithmetic.
__device__ __forceinline__ uint32_t silu_pair(float a0, float a1, uint32_t* zpair) {
  const __nv_bfloat162 z = __floats2bfloat162_rn(a0, a1);
  const __nv_bfloat162 half = __floats2bfloat162_rn(0.5f, 0.5f);
  const __nv_bfloat162 h = __hmul2(z, half);
  const uint32_t hb = *reinterpret_cast<const uint32_t*>(&h);
  const uint32_t tb = tanh_bf16x2(hb);
  const __nv_bfloat162 t = *reinterpret_cast<const __nv_bfloat162*>(&tb);
  const __nv_bfloat162 sg = __hfma2(t, half, half);
  const __nv_bfloat162 y = __hmul2(z, sg);
  if (zpair) *zpair = *reinterpret_cast<const uint32_t*>(&z);
  return *reinterpret_cast<const uint32_t*>(&y);
}

// Packs W_l into per-slice canonical K-major blocks: slice (l, c) element
// (n, k) at slice_off + (n/8)*1024 + (k/8)*128 + (n%8)*16 + (k%8)*2; K columns
// past fan_in are zero.
__global__ void pack_weights_kernel(const bf16* pb, const FwdArgs A, uint8_t* wpk) {
  for (int l = 0; l < A.layers; ++l) {
    const int N = A.fan_out[l], K = A.fan_in[l], nch = (K + kKC - 1) / kKC;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nch * N * 8; t += gridDim.x * blockDim.x) {
      const int c = t / (N * 8), rem = t - c * N * 8, n = rem >> 3, g = rem & 7;
      const int k = c * kKC + g * 8;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (k < K) v = *reinterpret_cast<const uint4*>(pb + A.w_off[l] + static_cast<size_t>(n) * K + k);
      *reinterpret_cast<uint4*>(wpk + A.slice_off[l][c] + (n >> 3) * kSBO + g * kLBO + (n & 7) * 16) = v;
    }
  }
}

__global__ void __launch_bounds__(kFwdThreads, 1) mlp_forward_fused_kernel(const FwdArgs A) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* act[2] = {smem, smem + kFwdAct};
  uint8_t* ring = smem + 2 * kFwdAct;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * kFwdAct + kFwdSlots * kFwdW);
  uint64_t* full = bars;              // [3] slice landed
  uint64_t* empty = bars + 3;         // [3] slice consumed by the tensor core
  uint64_t* acc_full = bars + 6;      // [2] tile's layer accumulated
  uint64_t* act_ready = bars + 8;     // [2] tile's layer input written (256 arrivals)
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 10);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 11);
  uint64_t* drain = bars + 12;        // completion of every MMA this CTA issued
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntiles = A.rows / kTM;
  const int npairs = (ntiles + 1) / 2;
  if (tid == 0) {
    for (int b = 0; b < 3; ++b) {
      umma::mbar_init(&full[b], 1);
      umma::mbar_init(&empty[b], 1);
    }
    for (int t = 0; t < 2; ++t) {
      umma::mbar_init(&acc_full[t], 1);
      umma::mbar_init(&act_ready[t], kFwdGroups * kTM);  // the tile's epilogue threads
    }
    umma::mbar_init(drain, 1);
    *abort_flag = 0;
  }
  if (warp == 1) umma::tmem_alloc(tslot, kFwdTmemCols);
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = *tslot;
  auto tiles_of = [&](int pair) { return 2 * pair + 1 < ntiles ? 2 : 1; };
  auto wait = [&](uint64_t* bar, uint32_t parity) -> bool {
    if (*abort_flag) return false;
    if (umma::mbar_wait(bar, parity, A.err, 3)) return true;
    *abort_flag = 1;
    return false;
  };

  if (warp == 0) {
    // ---- producer ----
    if (lane == 0) {
      uint32_t k = 0;
      bool ok = true;
      for (int pair = blockIdx.x; pair < npairs && ok; pair += gridDim.x) {
        const int nt = tiles_of(pair);
        for (int l = 0; l < A.layers && ok; ++l) {
          const int nch = (A.fan_in[l] + kKC - 1) / kKC;
          const uint32_t bytes = static_cast<uint32_t>(A.fan_out[l]) * (kKC * 2);
          for (int t = 0; t < nt && ok; ++t)
            for (int c = 0; c < nch; ++c, ++k) {
              const uint32_t slot = k % kFwdSlots;
              if (k >= kFwdSlots && !(ok = wait(&empty[slot], ((k / kFwdSlots) - 1) & 1u))) break;
              mbar_expect_tx(&full[slot], bytes);
              bulk_g2s(ring + slot * kFwdW, A.wpk + A.slice_off[l][c], bytes, &full[slot]);
            }
        }
      }
      // Drain (matters after an abort): the last copies issued into each slot
      // must have landed before the CTA's shared memory is released. In a normal
      // run their phases are already complete and these waits return at once.
      for (uint32_t j = k > static_cast<uint32_t>(kFwdSlots) ? k - kFwdSlots : 0u; j < k; ++j)
        umma::mbar_wait(&full[j % kFwdSlots], (j / kFwdSlots) & 1u, A.err, 3);
    }
  } else if (warp == 1) {
    // ---- MMA issuer ----
    if (lane == 0) {
      uint32_t k = 0, ph_act[2] = {0u, 0u};
      bool ok = true;
      for (int pair = blockIdx.x; pair < npairs && ok; pair += gridDim.x) {
        const int nt = tiles_of(pair);
        for (int l = 0; l < A.layers && ok; ++l) {
          const int N = A.fan_out[l], K = A.fan_in[l], nch = (K + kKC - 1) / kKC;
          const uint32_t idesc = umma::instr_desc_bf16_f32(kTM, N, false, false);
          for (int t = 0; t < nt && ok; ++t) {
            if (!(ok = wait(&act_ready[t], ph_act[t]))) break;
            ph_act[t] ^= 1u;
            umma::tc_fence_after();
            const uint32_t a0 = umma::smem_addr(act[t]);
            for (int c = 0; c < nch; ++c, ++k) {
              const uint32_t slot = k % kFwdSlots;
              if (!(ok = wait(&full[slot], (k / kFwdSlots) & 1u))) break;
              umma::tc_fence_after();
              const uint32_t bsm = umma::smem_addr(ring + slot * kFwdW);
              const int nks = min(kKC, K - c * kKC) / 16;
              for (int ks = 0; ks < nks; ++ks) {
                const uint64_t ad = umma::smem_desc(a0 + (c * (kKC / 8) + 2 * ks) * kLBO, kLBO, kFwdSboA);
                const uint64_t bd = umma::smem_desc(bsm + ks * 2 * kLBO, kLBO, kSBO);
                umma::mma_bf16(tmem + t * kTNmax, ad, bd, idesc, (c > 0 || ks > 0) ? 1u : 0u);
              }
              umma::mma_commit(&empty[slot]);
            }
            if (ok) umma::mma_commit(&acc_full[t]);
          }
        }
      }
      // Drain (matters after an abort): every MMA issued must have finished
      // writing TMEM before it is freed. In a normal run they all have.
      umma::mma_commit(drain);
      umma::mbar_wait(drain, 0u, A.err, 3);
    }
  } else {
    // ---- epilogue: 12 warps a tile; each warp one lane quarter (warp % 4, the
    // TMEM lanes it may read) and one group of 16-column chunks ----
    const int ew = warp - 2, t = ew / (4 * kFwdGroups), grp = (ew % (4 * kFwdGroups)) / 4, quarter = warp & 3;
    const int row = quarter * 32 + lane;
    const uint32_t tbase = tmem + (static_cast<uint32_t>(quarter * 32) << 16) + t * kTNmax;
    const int G = A.fan_in[0] / 8;
    auto load_x = [&](int pair) {
      const int m0 = (2 * pair + t) * kTM;
      for (int i = grp * kTM + row; i < kTM * G; i += kFwdGroups * kTM) {
        const int r = i / G, g = i - r * G;
        cp_async16(act[t] + (r >> 3) * kFwdSboA + g * kLBO + (r & 7) * 16,
                   A.x + static_cast<size_t>(m0 + r) * A.fan_in[0] + g * 8);
      }
      cp_async_commit();
      cp_async_wait_all();
      umma::fence_async_smem();
    };
    uint32_t ph_acc = 0;
    bool ok = true;
    int pair = blockIdx.x;
    if (pair < npairs && t < tiles_of(pair)) {
      load_x(pair);
      mbar_arrive(&act_ready[t]);
    }
    for (; pair < npairs && ok; pair += gridDim.x) {
      if (t >= tiles_of(pair)) break;
      const int m0 = (2 * pair + t) * kTM;
      for (int l = 0; l < A.layers && ok; ++l) {
        const int N = A.fan_out[l], nch16 = N / 16;
        const int cbeg = 16 * (grp * nch16 / kFwdGroups), cend = 16 * ((grp + 1) * nch16 / kFwdGroups);
        const float* bias = A.p + A.b_off[l];
        const bool last = l + 1 == A.layers;
        // this warp's first 16 biases, one per lane, fetched before the wait
        float bnext = lane < 16 ? __ldg(bias + cbeg + lane) : 0.0f;
        if (!(ok = wait(&acc_full[t], ph_acc))) break;
        ph_acc ^= 1u;
        umma::tc_fence_after();
        for (int c0 = cbeg; c0 < cend; c0 += 16) {
          uint32_t r[16];
          umma::tmem_ld16(tbase + static_cast<uint32_t>(c0), r);
          const float bl = bnext;  // lane j holds bias[c0 + j]
          if (c0 + 16 < cend) bnext = lane < 16 ? __ldg(bias + c0 + 16 + lane) : 0.0f;
          umma::tmem_wait_ld();
          float b[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) b[j] = __shfl_sync(0xffffffffu, bl, j);
          if (!last) {
            uint32_t y[8];
#pragma unroll
            for (int j = 0; j < 16; j += 2)
              y[j / 2] = silu_pair(__uint_as_float(r[j]) + b[j], __uint_as_float(r[j + 1]) + b[j + 1], nullptr);
            uint8_t* dst = act[t] + (row >> 3) * kFwdSboA + (c0 / 8) * kLBO + (row & 7) * 16;
            *reinterpret_cast<uint4*>(dst) = make_uint4(y[0], y[1], y[2], y[3]);
            *reinterpret_cast<uint4*>(dst + kLBO) = make_uint4(y[4], y[5], y[6], y[7]);
          } else {
            float* o = A.out + static_cast<size_t>(m0 + row) * N + c0;
#pragma unroll
            for (int j = 0; j < 16; j += 4)
              *reinterpret_cast<float4*>(o + j) =
                  make_float4(__uint_as_float(r[j]) + b[j], __uint_as_float(r[j + 1]) + b[j + 1],
                              __uint_as_float(r[j + 2]) + b[j + 2], __uint_as_float(r[j + 3]) + b[j + 3]);
          }
        }
        umma::tc_fence_before();
        if (!last) {
          umma::fence_async_smem();
          mbar_arrive(&act_ready[t]);
        } else {
          const int np = pair + static_cast<int>(gridDim.x);
          if (np < npairs && t < tiles_of(np)) {
            load_x(np);
            mbar_arrive(&act_ready[t]);
          }
        }
      }
    }
  }
  __syncthreads();
  if (warp == 1) {
    umma::tc_fence_after();
    umma::tmem_dealloc(tmem, kFwdTmemCols);
  }
}

}  // namespace mlp
}  // namespace ce

using ce::mlp::bf16;

struct ce_mlp {
  int device = 0;
  int in_dim = 0, hidden = 0, depth = 0, out_dim = 0;
  int layers = 0;
  std::vector<int> fan_in, fan_out;
  // FP32 master parameters, gradients and Adam state, laid out [W_0 b_0 W_1 b_1 ...].
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  bf16* pb = nullptr;  // BF16 copy of the weights (same layout)
  size_t n_params = 0;
  std::vector<size_t> w_off, b_off;
  // activations for up to max_batch rows
  uint64_t max_batch = 0;
  std::vector<bf16*> Z, H;  // per hidden layer: pre-activation, activation
  bf16 *dA = nullptr, *dB = nullptr;  // gradient ping-pong [B][max width]
  float* out = nullptr;               // [B][out_dim]
  bf16* dout = nullptr;               // [B][out_dim]
  float* loss = nullptr;              // device scalar
  int* err = nullptr;                 // device error flag
  uint64_t step = 0;
  // weights packed for the fused forward, refreshed when the parameters change
  uint8_t* wpk = nullptr;
  size_t wpk_bytes = 0;
  uint64_t param_version = 1, packed_version = 0;
  std::string msg;
};

namespace {

using namespace ce::mlp;

int set_err(ce_mlp* n, int code, const std::string& m) {
  if (n) n->msg = m;
  return code;
}

template <bool A, bool B>
int launch_gemm(ce_mlp* net, GemmArgs g, cudaStream_t s, int splits = 1) {
  if (g.M <= 0 || g.N <= 0 || g.K <= 0) return CE_OK;
  if (g.N % 16 != 0 || g.K % 8 != 0 || g.lda % 8 != 0 || g.ldb % 8 != 0)
    return set_err(net, CE_ERR_INVALID, "umma gemm: N must be a multiple of 16, K and leading dims of 8");
  const auto fn = &umma_gemm_kernel<A, B>;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes) != cudaSuccess)
    return set_err(net, CE_ERR_CUDA, "cudaFuncSetAttribute");
  int per = (g.K + splits - 1) / splits;
  per = ((per + kKC - 1) / kKC) * kKC;
  g.k_split = per;
  const int z = (g.K + per - 1) / per;
  g.err = net->err;
  dim3 grid((g.M + kTM - 1) / kTM, (g.N + kTNmax - 1) / kTNmax, z);
  fn<<<grid, 128, kSmemBytes, s>>>(g);
  return cudaGetLastError() == cudaSuccess ? CE_OK : set_err(net, CE_ERR_CUDA, "umma gemm launch");
}

GemmArgs args0() {
  GemmArgs g;
  std::memset(&g, 0, sizeof g);
  return g;
}

int forward(ce_mlp* net, const bf16* x, uint64_t B, cudaStream_t s) {
  const bf16* in = x;
  int in_ld = net->in_dim;
  for (int l = 0; l < net->layers; ++l) {
    GemmArgs g = args0();
    g.A = in;
    g.lda = in_ld;
    g.B = net->pb + net->w_off[l];
    g.ldb = net->fan_in[l];
    g.M = static_cast<int>(B);
    g.N = net->fan_out[l];
    g.K = net->fan_in[l];
    g.bias = net->p + net->b_off[l];
    if (l + 1 < net->layers) {
      g.epi = kEpiFwdAct;
      g.Zout = net->Z[l];
      g.ldz = net->hidden;
      g.Y = net->H[l];
      g.ldy = net->hidden;
    } else {
      g.epi = kEpiFwdLinearF32;
      g.C = net->out;
      g.ldc = net->out_dim;
    }
    const int rc = launch_gemm<false, false>(net, g, s);
    if (rc != CE_OK) return rc;
    in = net->H[l];
    in_ld = net->hidden;
  }
  return CE_OK;
}

// Gradients of the mean-squared loss into net->g (zeroed here).
int backward(ce_mlp* net, const bf16* x, const float* target, const float* w, uint64_t B, cudaStream_t s) {
  cudaMemsetAsync(net->g, 0, net->n_params * sizeof(float), s);
  cudaMemsetAsync(net->loss, 0, sizeof(float), s);
  // weight sum on the host side of the contract: callers pass normalised weights.
  const int n_total = static_cast<int>(B) * net->out_dim;
  mse_grad_kernel<<<256, 256, 0, s>>>(net->out, target, w, 1.0f, n_total, net->dout, net->loss);
  const int L = net->layers;
  const int splits = static_cast<int>((B + 511) / 512);
  const bf16* dcur = net->dout;  // gradient w.r.t. the current layer's pre-activation
  int dcur_ld = net->out_dim;
  for (int l = L - 1; l >= 0; --l) {
    const bf16* in = l == 0 ? x : net->H[l - 1];
    const int in_ld = l == 0 ? net->in_dim : net->hidden;
    const int fo = net->fan_out[l], fi = net->fan_in[l];
    // dW_l = dcur^T in  ([fo][fi]); use the transposed form when fo < 128 rows.
    GemmArgs g = args0();
    if (fo >= kTM) {
      g.A = dcur;  // A(m = o, k = b) = dcur[b][o]: MN-major
      g.lda = dcur_ld;
      g.B = in;  // B(n = i, k = b) = in[b][i]: MN-major
      g.ldb = in_ld;
      g.M = fo;
      g.N = fi;
      g.K = static_cast<int>(B);
      g.epi = kEpiAtomicF32;
      g.C = net->g + net->w_off[l];
      g.ldc = fi;
    } else {
      g.A = in;  // A(m = i, k = b) = in[b][i]
      g.lda = in_ld;
      g.B = dcur;  // B(n = o, k = b) = dcur[b][o]
      g.ldb = dcur_ld;
      g.M = fi;
      g.N = fo;
      g.K = static_cast<int>(B);
      g.epi = kEpiAtomicF32T;
      g.C = net->g + net->w_off[l];
      g.ldc = fi;
    }
    int rc = launch_gemm<true, true>(net, g, s, splits);
    if (rc != CE_OK) return rc;
    colsum_kernel<<<dim3((fo + 127) / 128, static_cast<unsigned>((B + kColRows - 1) / kColRows)), 128, 0, s>>>(
        dcur, static_cast<int>(B), fo, dcur_ld, net->g + net->b_off[l]);
    if (l == 0) break;
    // d(pre-activation of layer l-1) = (dcur W_l) * silu'(Z_{l-1})
    bf16* dnext = (dcur == net->dA) ? net->dB : net->dA;
    GemmArgs h = args0();
    h.A = dcur;  // [B][fo], K-major
    h.lda = dcur_ld;
    h.B = net->pb + net->w_off[l];  // B(n = i, k = o) = W[o][i]: MN-major
    h.ldb = fi;
    h.M = static_cast<int>(B);
    h.N = fi;
    h.K = fo;
    h.epi = kEpiBwdAct;
    h.Zin = net->Z[l - 1];
    h.ldz = net->hidden;
    h.Y = dnext;
    h.ldy = net->hidden;
    rc = launch_gemm<false, true>(net, h, s);
    if (rc != CE_OK) return rc;
    dcur = dnext;
    dcur_ld = net->hidden;
  }
  return cudaGetLastError() == cudaSuccess ? CE_OK : set_err(net, CE_ERR_CUDA, "backward launch");
}

// The fused serving forward holds a 128-row tile of every layer's input in
// shared memory (width <= 256) and splits each layer's columns over two warp
// groups in 16-column TMEM loads (width a multiple of 32).
bool fused_eligible(const ce_mlp* n) {
  if (n->layers > ce::mlp::kFwdMaxLayers || n->in_dim > ce::mlp::kFwdKmax || n->in_dim % 8) return false;
  for (int l = 0; l < n->layers; ++l)
    if (n->fan_out[l] % 32 || n->fan_out[l] > ce::mlp::kTNmax) return false;
  return n->n_params < (1ull << 31);
}

int check_err_flag(ce_mlp* net, cudaStream_t s) {
  int h = 0;
  if (cudaMemcpyAsync(&h, net->err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return set_err(net, CE_ERR_CUDA, "MLP kernels failed");
  if (h != 0) return set_err(net, CE_ERR_CUDA, "MLP tensor-core wait timed out");
  return CE_OK;
}

}  // namespace

extern "C" {

int ce_mlp_create(ce_mlp** out, int device, int in_dim, int hidden, int depth, int out_dim, uint64_t max_batch,
                  uint64_t seed) {
  if (!out) return CE_ERR_INVALID;
  *out = nullptr;
  if (in_dim <= 0 || in_dim % 16 || hidden <= 0 || hidden % 16 || hidden > 256 || depth < 1 || out_dim <= 0 ||
      out_dim % 16 || out_dim > 256 || max_batch == 0 || max_batch % 128)
    return CE_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return CE_ERR_NO_DEVICE;
  ce_mlp* n = new ce_mlp();
  n->device = device;
  n->in_dim = in_dim;
  n->hidden = hidden;
  n->depth = depth;
  n->out_dim = out_dim;
  n->layers = depth + 1;
  n->max_batch = max_batch;
  for (int l = 0; l < n->layers; ++l) {
    n->fan_in.push_back(l == 0 ? in_dim : hidden);
    n->fan_out.push_back(l + 1 < n->layers ? hidden : out_dim);
  }
  size_t off = 0;
  for (int l = 0; l < n->layers; ++l) {
    n->w_off.push_back(off);
    off += static_cast<size_t>(n->fan_in[l]) * n->fan_out[l];
    n->b_off.push_back(off);
    off += n->fan_out[l];
  }
  n->n_params = off;
  bool okm = cudaMalloc(&n->p, off * 4) == cudaSuccess && cudaMalloc(&n->g, off * 4) == cudaSuccess &&
             cudaMalloc(&n->m, off * 4) == cudaSuccess && cudaMalloc(&n->v, off * 4) == cudaSuccess &&
             cudaMalloc(&n->pb, off * 2) == cudaSuccess && cudaMalloc(&n->loss, 4) == cudaSuccess &&
             cudaMalloc(&n->err, 4) == cudaSuccess &&
             cudaMalloc(&n->out, max_batch * out_dim * 4) == cudaSuccess &&
             cudaMalloc(&n->dout, max_batch * out_dim * 2) == cudaSuccess &&
             cudaMalloc(&n->dA, max_batch * hidden * 2) == cudaSuccess &&
             cudaMalloc(&n->dB, max_batch * hidden * 2) == cudaSuccess;
  for (int l = 0; l + 1 < n->layers && okm; ++l) {
    bf16 *z = nullptr, *h = nullptr;
    okm = cudaMalloc(&z, max_batch * hidden * 2) == cudaSuccess && cudaMalloc(&h, max_batch * hidden * 2) == cudaSuccess;
    n->Z.push_back(z);
    n->H.push_back(h);
  }
  if (!okm) {
    ce_mlp_destroy(n);
    return CE_ERR_CUDA;
  }
  // He-uniform init for SiLU layers, smaller for the output layer; zero biases.
  std::vector<float> h(off, 0.0f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < n->layers; ++l) {
    const float lim = (l + 1 < n->layers ? std::sqrt(6.0f / n->fan_in[l]) : 0.1f * std::sqrt(3.0f / n->fan_in[l]));
    std::uniform_real_distribution<float> u(-lim, lim);
    for (size_t i = 0; i < static_cast<size_t>(n->fan_in[l]) * n->fan_out[l]; ++i) h[n->w_off[l] + i] = u(rng);
  }
  const int rc = ce_mlp_set_params(n, h.data());
  cudaMemset(n->m, 0, off * 4);
  cudaMemset(n->v, 0, off * 4);
  cudaMemset(n->err, 0, 4);
  if (rc != CE_OK) {
    ce_mlp_destroy(n);
    return rc;
  }
  *out = n;
  return CE_OK;
}

void ce_mlp_destroy(ce_mlp* n) {
  if (!n) return;
  cudaSetDevice(n->device);
  for (void* p : {static_cast<void*>(n->p), static_cast<void*>(n->g), static_cast<void*>(n->m),
                  static_cast<void*>(n->v), static_cast<void*>(n->pb), static_cast<void*>(n->loss),
                  static_cast<void*>(n->err), static_cast<void*>(n->out), static_cast<void*>(n->dout),
                  static_cast<void*>(n->dA), static_cast<void*>(n->dB)})
    if (p) cudaFree(p);
  if (n->wpk) cudaFree(n->wpk);
  for (bf16* z : n->Z) cudaFree(z);
  for (bf16* h : n->H) cudaFree(h);
  delete n;
}

const char* ce_mlp_last_error(const ce_mlp* n) { return n ? n->msg.c_str() : "null network"; }

uint64_t ce_mlp_param_count(const ce_mlp* n) { return n ? n->n_params : 0; }

int ce_mlp_set_params(ce_mlp* n, const float* host) {
  if (!n || !host) return CE_ERR_INVALID;
  cudaSetDevice(n->device);
  if (cudaMemcpy(n->p, host, n->n_params * 4, cudaMemcpyHostToDevice) != cudaSuccess) return CE_ERR_CUDA;
  ce::mlp::f32_to_bf16_kernel<<<256, 256>>>(n->p, n->pb, static_cast<int>(n->n_params));
  ++n->param_version;
  return cudaDeviceSynchronize() == cudaSuccess ? CE_OK : CE_ERR_CUDA;
}

int ce_mlp_get_params(const ce_mlp* n, float* host) {
  if (!n || !host) return CE_ERR_INVALID;
  cudaSetDevice(n->device);
  return cudaMemcpy(host, n->p, n->n_params * 4, cudaMemcpyDeviceToHost) == cudaSuccess ? CE_OK : CE_ERR_CUDA;
}

int ce_mlp_forward_layered(ce_mlp* n, const void* x, uint64_t B, float* out, void* stream) {
  if (!n || !x || !out || B == 0 || B % 128 || B > n->max_batch)
    return set_err(n, CE_ERR_INVALID, "ce_mlp_forward_layered: B must be a positive multiple of 128 up to max_batch");
  cudaSetDevice(n->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = forward(n, static_cast<const bf16*>(x), B, s);
  if (rc != CE_OK) return rc;
  if (cudaMemcpyAsync(out, n->out, B * n->out_dim * 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return set_err(n, CE_ERR_CUDA, "copy out");
  return CE_OK;
}

int ce_mlp_forward(ce_mlp* n, const void* x, uint64_t B, float* out, void* stream) {
  if (!n || !x || !out || B == 0 || B % 128) return set_err(n, CE_ERR_INVALID, "ce_mlp_forward: B must be a positive multiple of 128");
  if (!fused_eligible(n)) {
    if (B > n->max_batch) return set_err(n, CE_ERR_INVALID, "ce_mlp_forward: B exceeds max_batch");
    return ce_mlp_forward_layered(n, x, B, out, stream);
  }
  if (B > (1ull << 30)) return set_err(n, CE_ERR_INVALID, "ce_mlp_forward: B above 2^30 rows");
  cudaSetDevice(n->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  using namespace ce::mlp;
  FwdArgs a{};
  a.x = static_cast<const bf16*>(x);
  a.p = n->p;
  a.out = out;
  a.rows = static_cast<int>(B);
  a.layers = n->layers;
  size_t off = 0;
  for (int l = 0; l < n->layers; ++l) {
    a.fan_in[l] = n->fan_in[l];
    a.fan_out[l] = n->fan_out[l];
    a.w_off[l] = static_cast<int>(n->w_off[l]);
    a.b_off[l] = static_cast<int>(n->b_off[l]);
    for (int c = 0; c * kKC < n->fan_in[l]; ++c) {
      a.slice_off[l][c] = static_cast<int>(off);
      off += static_cast<size_t>(n->fan_out[l]) * kKC * 2;
    }
  }
  a.err = n->err;
  if (off > n->wpk_bytes) {
    if (n->wpk) cudaFree(n->wpk);
    n->wpk = nullptr;
    n->wpk_bytes = 0;
    if (cudaMalloc(&n->wpk, off) != cudaSuccess) return set_err(n, CE_ERR_CUDA, "cudaMalloc(packed weights)");
    n->wpk_bytes = off;
    n->packed_version = 0;
  }
  a.wpk = n->wpk;
  if (n->packed_version != n->param_version) {
    pack_weights_kernel<<<128, 256, 0, s>>>(n->pb, a, n->wpk);
    n->packed_version = n->param_version;
  }
  if (cudaFuncSetAttribute(mlp_forward_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmem) !=
      cudaSuccess)
    return set_err(n, CE_ERR_CUDA, "cudaFuncSetAttribute(fused forward)");
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, n->device);
  const int pairs = static_cast<int>((B / kTM + 1) / 2);
  mlp_forward_fused_kernel<<<pairs < sms ? pairs : sms, kFwdThreads, kFwdSmem, s>>>(a);
  return cudaGetLastError() == cudaSuccess ? CE_OK : set_err(n, CE_ERR_CUDA, "fused forward launch");
}

int ce_mlp_gradients(ce_mlp* n, const void* x, const float* target, const float* weight, uint64_t B, float* loss,
                     float* grads_host, void* stream) {
  if (!n || !x || !target || !weight || B == 0 || B % 128 || B > n->max_batch)
    return set_err(n, CE_ERR_INVALID, "ce_mlp_gradients: B must be a positive multiple of 128 up to max_batch");
  cudaSetDevice(n->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = forward(n, static_cast<const bf16*>(x), B, s);
  if (rc == CE_OK) rc = backward(n, static_cast<const bf16*>(x), target, weight, B, s);
  if (rc != CE_OK) return rc;
  rc = check_err_flag(n, s);
  if (rc != CE_OK) return rc;
  if (loss && cudaMemcpy(loss, n->loss, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return CE_ERR_CUDA;
  if (grads_host && cudaMemcpy(grads_host, n->g, n->n_params * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return CE_ERR_CUDA;
  return CE_OK;
}

int ce_mlp_train_step(ce_mlp* n, const void* x, const float* target, const float* weight, uint64_t B, float lr,
                      float* loss_dev_accum, void* stream) {
  if (!n || !x || !target || !weight || B == 0 || B % 128 || B > n->max_batch)
    return set_err(n, CE_ERR_INVALID, "ce_mlp_train_step: B must be a positive multiple of 128 up to max_batch");
  cudaSetDevice(n->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = forward(n, static_cast<const bf16*>(x), B, s);
  if (rc == CE_OK) rc = backward(n, static_cast<const bf16*>(x), target, weight, B, s);
  if (rc != CE_OK) return rc;
  ++n->step;
  ++n->param_version;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - std::pow(b1, static_cast<float>(n->step));
  const float c2 = 1.0f - std::pow(b2, static_cast<float>(n->step));
  ce::mlp::adam_kernel<<<512, 256, 0, s>>>(n->p, n->g, n->m, n->v, n->pb, static_cast<int>(n->n_params), lr, b1, b2,
                                           1e-8f, c1, c2);
  if (loss_dev_accum) {
    // accumulate this step's loss on the device (no host sync per step)
    cudaMemcpyAsync(loss_dev_accum, n->loss, 4, cudaMemcpyDeviceToDevice, s);
  }
  return cudaGetLastError() == cudaSuccess ? CE_OK : set_err(n, CE_ERR_CUDA, "adam launch");
}

int ce_mlp_shape(const ce_mlp* n, int* in_dim, int* hidden, int* depth, int* out_dim, uint64_t* max_batch) {
  if (!n) return CE_ERR_INVALID;
  if (in_dim) *in_dim = n->in_dim;
  if (hidden) *hidden = n->hidden;
  if (depth) *depth = n->depth;
  if (out_dim) *out_dim = n->out_dim;
  if (max_batch) *max_batch = n->max_batch;
  return CE_OK;
}

int ce_mlp_check(ce_mlp* n, void* stream) {
  if (!n) return CE_ERR_INVALID;
  return check_err_flag(n, static_cast<cudaStream_t>(stream));
}

// Raw tensor-core GEMM entry for unit tests: C[M][N] (f32) = A * B^T with A
// given K-major [M][K] or MN-major [K][M], B likewise ([N][K] or [K][N]).
int ce_umma_gemm_f32(const void* A, int a_mn, const void* B, int b_mn, int M, int N, int K, float* C, int* err_dev,
                     void* stream) {
  if (!A || !B || !C || M <= 0 || N <= 0 || K <= 0 || N % 16 || K % 8 || M % 8) return CE_ERR_INVALID;
  ce_mlp tmp;
  tmp.err = err_dev;
  GemmArgs g = args0();
  g.A = static_cast<const bf16*>(A);
  g.lda = a_mn ? M : K;
  g.B = static_cast<const bf16*>(B);
  g.ldb = b_mn ? N : K;
  g.M = M;
  g.N = N;
  g.K = K;
  g.epi = kEpiAtomicF32;
  g.C = C;
  g.ldc = N;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(C, 0, static_cast<size_t>(M) * N * 4, s) != cudaSuccess) return CE_ERR_CUDA;
  if (a_mn && b_mn) return launch_gemm<true, true>(&tmp, g, s, (K + 511) / 512);
  if (a_mn) return launch_gemm<true, false>(&tmp, g, s, (K + 511) / 512);
  if (b_mn) return launch_gemm<false, true>(&tmp, g, s, (K + 511) / 512);
  return launch_gemm<false, false>(&tmp, g, s, (K + 511) / 512);
}

}  // extern "C"
