// Shared definitions for the deltamic_b200 CUDA library: status codes, cell
// descriptors for batched launches, and the sm_90+/sm_100a PTX used to stage
// tiles in shared memory with the bulk-copy (TMA) engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/deltamic_b200.h"

namespace dm {

// ---------------------------------------------------------------------------
// Records held in HBM

// One face, 64 bytes, 16-byte aligned so a tile of faces is one bulk copy.
struct alignas(16) FaceRec {
  uint32_t Ua[3], Ub[3], Uc[3];  // fixed-point positions of the three vertices
  float hab[3], hbc[3];          // half-unit edge vectors (see pair_math.cuh)
  float area_coeff;              // |(b-a)x(c-a)|/2 * Faces_coeff
};
static_assert(sizeof(FaceRec) == 64, "FaceRec layout");

// One narrow-band frequency with its cotangent, 32 bytes (backward input).
struct alignas(16) XiRec {
  int32_t mi[3];
  float g_re;
  float mf[3];
  float g_im;
};
static_assert(sizeof(XiRec) == 32, "XiRec layout");

// A frequency off the grid (explicit xi list), 48 bytes: the XiRec fields with
// the real m_d = xi_d L_d / pi in mf, its nearest integer in mi and the
// remainder m_d - mi_d in fr (split phase, pair_math.cuh).
struct alignas(16) XiRecOff {
  int32_t mi[3];
  float g_re;
  float mf[3];
  float g_im;
  float fr[3];
  float pad;
};
static_assert(sizeof(XiRecOff) == 48, "XiRecOff layout");

// Per-cell description of a batched launch.  A single mesh is a batch of one.
struct CellDesc {
  double lo[3];       // box lower corner (box_size[:,0])
  double len[3];      // box extents
  int32_t n[3];       // box_shape
  int32_t nv, nt, nband;
  int32_t ne;         // frequencies evaluated: band[0, ne) (half the band if herm)
  int32_t herm;       // band closed under xi -> -xi (DM_BAND_HERMITIAN)
  int64_t v_off;      // first vertex in the concatenated vertex array
  int64_t f_off;      // first face in the concatenated face arrays
  int64_t b_off;      // first band entry in the concatenated band arrays
  int64_t grid_off;   // first element of this cell's dense grid
  int64_t fpart_off;  // forward partials (complex elements)
  int64_t bpart_off;  // backward partials (floats)
  int32_t fsplit;     // forward: face splits (partial sums per frequency)
  int32_t fchunk;     // forward: faces per split
  int32_t xtiles;     // forward: frequency tiles
  int32_t bchunks;    // backward: frequency chunks
  int32_t bxchunk;    // backward: frequencies per chunk
  int32_t fblocks;    // backward: face blocks
  int32_t fwd_item0;  // first forward work item of this cell
  int32_t bwd_item0;  // first backward work item of this cell
  int32_t face_blk0;  // first 256-face block of this cell (element-wise kernels)
  int32_t band_blk0;  // first 256-frequency block of this cell
};

// Cells of a launch: either one descriptor passed by value, or a device array.
struct Cells {
  const CellDesc* p;
  int32_t n;
  CellDesc one;
};

#if defined(__CUDACC__)
__device__ __forceinline__ CellDesc cell_get(const Cells& c, int i) { return c.p ? c.p[i] : c.one; }

// Index of the cell owning global item ``item`` given per-cell first items.
template <typename F>
__device__ __forceinline__ int cell_find(const Cells& c, int64_t item, F first) {
  if (!c.p) return 0;
  int lo = 0, hi = c.n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if ((int64_t)first(c.p[mid]) <= item) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ void set_error(int* err, int code) {
  if (err) atomicOr(err, code);
}

// ---------------------------------------------------------------------------
// Bulk-copy (TMA) staging into shared memory with mbarrier completion.
// Plain CTA-local copies: every copy lands in the issuing block's own shared
// memory, from this GPU's global memory.

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Global -> shared bulk copy; ``bytes`` a multiple of 16, both addresses 16-byte aligned.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after ``kWaitLimit`` polls, records DM_ERR_TIMEOUT and
// returns false so the kernel can leave instead of hanging the GPU.
// try_wait with a suspend-time hint: the thread may sleep up to ``ns`` nanoseconds
// for the phase to complete instead of spinning on issue slots.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity, uint32_t ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
      : "memory");
  return ok != 0;
}

// Bounded sleeping wait for a copy issued just before: at most kSleepTries tries
// of up to kSleepNs each (about 1.3 s in all), then DM_ERR_TIMEOUT and false.
constexpr uint32_t kSleepTries = 1u << 16;
constexpr uint32_t kSleepNs = 20000;
__device__ __forceinline__ bool mbar_wait_sleep_bounded(uint64_t* bar, uint32_t parity,
                                                        int* err,
                                                        uint32_t tries = kSleepTries) {
  for (uint32_t i = 0; i < tries; ++i)
    if (mbar_try_wait_sleep(bar, parity, kSleepNs)) return true;
  set_error(err, DM_ERR_TIMEOUT);
  return false;
}

constexpr uint32_t kWaitLimit = 1u << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err,
                                                  uint32_t limit = kWaitLimit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  set_error(err, DM_ERR_TIMEOUT);
  return false;
}
#endif

}  // namespace dm
