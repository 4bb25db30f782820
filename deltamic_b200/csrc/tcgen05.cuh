// Fifth-generation tensor-core primitives (sm_100a): TMEM allocation, shared-memory
// matrix descriptors, tcgen05.mma of kind::f16 (BF16 x BF16 -> FP32) issued by one
// thread, completion through tcgen05.commit on an mbarrier, and TMEM -> register
// loads.  Single-CTA forms only (cta_group::1), no multicast anywhere.
//
// Operand layout used by this library: "K-major, no swizzle".  A tile of R rows x
// 32 BF16 reduction elements is stored as 8-row x 16-byte core matrices (128
// contiguous bytes each); the four core matrices of one 8-row group along the
// reduction are adjacent (leading byte offset 128) and 8-row groups are 512 bytes
// apart (stride byte offset).  Element (r, k) of the tile is at element offset
// kmaj32_off(r, k).  One MMA consumes 16 reduction elements, i.e. two core
// matrices along K; the second MMA of a 32-wide stage starts 256 bytes further.
#pragma once
#include <stdint.h>

#include "dm_common.cuh"

namespace dm {
namespace tc {

__device__ __forceinline__ int kmaj32_off(int r, int k) {
  return (r >> 3) * 256 + (k >> 3) * 64 + (r & 7) * 8 + (k & 7);
}

constexpr uint32_t kLbo = 128;  // bytes between core matrices adjacent along K
constexpr uint32_t kSbo = 512;  // bytes between 8-row groups

// Shared-memory matrix descriptor: start address, leading and stride byte offsets
// (all >> 4), descriptor version 1 (bit 46), base offset 0, no swizzle (bits 61-63).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((kLbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((kSbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), A and B
// BF16 (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bit 17,
// M >> 4 at bit 24.
template <int M, int N>
__host__ __device__ constexpr uint32_t idesc_bf16_f32() {
  static_assert(M == 128, "one-CTA tiles of 128 rows");
  static_assert(N % 16 == 0 && N >= 16 && N <= 256, "M = 128 needs N a multiple of 16 in [16, 256]");
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Columns to allocate for an N-column FP32 accumulator (a power of two, >= 32).
template <int N>
__host__ __device__ constexpr int tmem_cols() {
  return N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
}

// Whole warp: allocate ``ncols`` TMEM columns, address written to *slot (shared).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// Whole warp (the allocating one).
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A[smem] B[smem]^T over 16 reduction elements; one thread issues.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, bool accumulate) {
  const uint32_t mask0 = 0, acc = accumulate ? 1u : 0u;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(
          d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(mask0)
      : "memory");
}

// The mbarrier completes one phase when every MMA this thread issued so far is done.
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// Warp-collective: lane i receives 16 consecutive FP32 columns of TMEM lane
// (lane field of taddr) + i; the wait is in the same statement, so the registers
// are complete when it returns.
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// The same for 8 consecutive columns.
__device__ __forceinline__ void ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int j = 0; j < 8; ++j) v[j] = __uint_as_float(r[j]);
}

}  // namespace tc
}  // namespace dm
