// umma.cuh -- Blackwell (sm_100a) 5th-generation tensor-core helpers in inline
// PTX: tcgen05.mma (kind::f16, BF16 in, FP32 accumulate in tensor memory),
// tcgen05.commit to an mbarrier, TMEM allocation and loads, and the shared-
// memory / instruction descriptors.
//
// Descriptor layouts follow the PTX ISA's tcgen05 "matrix descriptor" and
// "instruction descriptor" definitions (the same fields CUTLASS encodes in
// cute/arch/mma_sm100_desc.hpp):
//   instruction descriptor (32 bit): [4,6) D format (1 = F32), [7,10) A format
//   (1 = BF16), [10,13) B format, [15] A major (0 = K, 1 = MN), [16] B major,
//   [17,23) N >> 3, [24,29) M >> 4.
//   shared-memory descriptor (64 bit): [0,14) start address >> 4, [16,30)
//   leading-dimension byte offset >> 4, [32,46) stride-dimension byte offset
//   >> 4, [46,48) version (1 on sm_100), [61,64) layout (0 = no swizzle).
// Operands are staged in the no-swizzle canonical layout: "core matrices" of
// 8 rows x 16 bytes (8 bf16 along the operand's contiguous dimension) stored
// contiguously; core matrices adjacent in K are LBO bytes apart, adjacent in
// M/N SBO bytes apart (for a K-major operand the 8 rows run along M/N, for an
// MN-major operand along K).
//
// Every wait is bounded: a wait that runs out records an error code in global
// memory and returns false, so the kernel can release its tensor memory and
// exit instead of hanging the GPU.
#pragma once

#include <cstdint>

namespace ce {
namespace umma {

constexpr uint32_t kWaitSpins = 1u << 18;  // ~4 us per poll on B200: about one second

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint32_t instr_desc_bf16_f32(int M, int N, bool a_mn, bool b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(a_mn) << 15) |
         (static_cast<uint32_t>(b_mn) << 16) | (static_cast<uint32_t>(N >> 3) << 17) |
         (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= static_cast<uint64_t>(1u) << 46;  // descriptor version for sm_100
  return d;                              // layout type 0: no swizzle
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Wait for the phase with parity `parity` of `bar` to complete; bounded by
// `spins` polls, after which `code` is recorded in *err and false returned.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code,
                                          uint32_t spins = kWaitSpins) {
  const uint32_t a = smem_addr(bar);
  for (uint32_t i = 0; i < spins; ++i) {
    uint32_t done = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  if (err) atomicExch(err, code);
  return false;
}

// Make this thread's generic-proxy shared-memory writes visible to the tensor
// core (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// One full warp: allocate `ncols` TMEM columns (power of two >= 32); the base
// address is written to *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T for one K = 16 slice; issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      :
      : "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive on `bar` once every previously issued tcgen05.mma of this thread has
// completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

// 32 lanes x 16 columns of 32-bit TMEM values into registers (one row per thread).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

}  // namespace umma
}  // namespace ce
