// Footprint convolution kernels (included by conv.cu): the forward, data gradient
// and weight gradient of the 3x3x3 stride-2 convolution for the encoder's middle
// layers (Ci = 16 -> Co = 32 and Ci = 32 -> Co = 64), with the MMA operands read
// straight from a tile's input footprint in shared memory -- no im2col copy.
//
// A tile is 16 "lines" of 8 voxels along the fastest spatial axis (128 rows, the
// MMA's M).  Its input footprint is staged once (zero outside the volume, which is
// the padding), channel groups of eight (16 bytes) as the unit, laid out so that for
// every tap the 8 rows of a core matrix are 8 consecutive 16-byte chunks and the 16
// lines are a uniform stride apart.  A tap is then only a start address: the
// shared-memory matrix descriptor of tap t points into the footprint with the line
// stride as its stride byte offset and the channel-group stride as its leading byte
// offset.  The forward and the data gradient stage the footprint and the weight
// image with TMA boxes (layouts at FpWeights, FpFwd and FpDgrad below); the weight
// gradient, whose layout interleaves rows and channel groups, with cp.async.
//
// Data gradient, tile of input voxels (b, 2 jd + pd, 2 (jh0 + l) + ph, 2 (jw0 + i) +
// pw) for all eight parity classes (pd, ph, pw): per axis, parity 0 takes tap 1 from
// output j and parity 1 taps 0 and 2 from outputs j + 1 and j, so the tile needs dP
// at outputs (jd + dd, jh0 + hh, jw0 + ww), dd < 2, hh < 17, ww < 9.  Each class
// accumulates in its own TMEM columns (class * Ci), the 27 taps are each issued once.
//
// Weight gradient, per block one input plane kd (blockIdx.y) and a run of forward
// tiles (blockIdx.x): dW[(kd, kh, kw, ci), co] = sum_m x[m through the tap][ci]
// dP[m, co].  The accumulator rows are (r, ci) with r = input row offset 0..16/C8-1
// (rows r < 3 are the taps kh = r; the others are never stored), one accumulator
// per kw, N = Co, K = the tile's output voxels.  The footprint plane of a tile is
// chunk ((r * C8 + c8) * 2 + par) * 9 + j (rows of one input row's channel groups
// adjacent), read as the MN-major A operand: 8 voxels of a line are a core
// matrix's 8 reduction rows, channel groups then input rows are 288 bytes apart
// along M, and lines (two input rows) are 36 C8 chunks apart along K.  dP of the
// tile is the MN-major B operand, chunk co8 * 128 + voxel.  Block kd = 1 also sums
// dP against a block of ones (the bias gradient).
#pragma once

namespace dm {

__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// Waits for an MMA commit with only thread 0 sleeping on the barrier (every
// thread polling it spends issue slots the other blocks on the SM need); after the
// block barrier each other thread confirms the completed phase with one test.
// ``mine`` folds a thread's own failure into the (block-uniform) answer.
__device__ __forceinline__ bool mbar_wait_block(uint64_t* bar, uint32_t parity, int* err,
                                                bool mine = true) {
  int ok = mine ? 1 : 0;
  if (threadIdx.x == 0) ok = (mbar_wait_sleep_bounded(bar, parity, err) && mine) ? 1 : 0;
  ok = __syncthreads_and(ok);
  if (ok && threadIdx.x != 0) ok = mbar_wait_bounded(bar, parity, err) ? 1 : 0;
  return __syncthreads_and(ok) != 0;  // the same answer in every thread
}

__device__ __forceinline__ void mbar_arrive1(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Named barrier ``id`` over ``n`` threads that also ANDs a flag across them (every
// participant leaves with the same answer).
__device__ __forceinline__ bool named_bar_and(int id, int n, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id), "r"(n)
      : "memory");
  return r != 0;
}

// Tensor-map (TMA) box loads from this GPU's global memory into shared memory,
// completing on an mbarrier (no multicast).  Coordinates innermost first; the
// innermost one (a channel) is a multiple of 8 BF16 (16 bytes); the others may be
// negative or past the extent (those elements read zero).
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, int c3, int c4, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

// Shared-memory matrix descriptor with explicit leading / stride byte offsets (bytes,
// multiples of 16), no swizzle, descriptor version 1.
__device__ __forceinline__ uint64_t fp_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Threads of a footprint block: eight warps; warp w reads accumulator lanes
// 32 (w % 4) .. + 31 (its TMEM lane quarter) and the column half w / 4.
constexpr int kFpThreads = 256;

// Weight image, loaded by TMA as CO / 8 boxes {8 co, CI ci, 27 taps} of W viewed as
// [tap][ci][co]: chunk (co8, tap, ci) = W[tap * CI + ci, 8 co8 .. 8 co8 + 7] at
// (co8 * 27 + tap) * CI + ci.  It is the forward's MN-major B (N = co: groups of 8
// co 27 CI chunks apart, K = ci: rows 16 bytes apart, groups of 8 ci 128 bytes
// apart) and the data gradient's K-major B (N = ci rows, K = co: groups 27 CI
// chunks apart).
template <int CI, int CO>
struct FpWeights {
  static constexpr int kBoxBytes = 8 * CI * 27 * 2;
  static constexpr int kBytes = (CO / 8) * kBoxBytes;
  static_assert(kBoxBytes % 128 == 0, "weight boxes 128-byte aligned");
};

template <int CI, int CO>
__device__ __forceinline__ void fp_tma_weights(uint8_t* wimg, const CUtensorMap* wmap,
                                               uint64_t* bar) {
#pragma unroll
  for (int co8 = 0; co8 < CO / 8; ++co8)
    tma_load_3d(wimg + co8 * FpWeights<CI, CO>::kBoxBytes, wmap, co8 * 8, 0, 0, bar);
}

// Forward footprint (TMA): box (c8, par) = x[b, 2 od - 1 + kd, 2 oh0 - 1 + r,
// 2 ow0 - 1 + par + 2 j, 8 c8 .. + 7], kd < 3, r < HR, j < 9 (a W traversal stride
// of 2 de-interleaves the parities), chunk ((kd * HR + r) * 9 + j) of the box; boxes
// (c8 * 2 + par) are kBlk chunks apart (128-byte aligned).  Tap (kd, kh, kw) of
// output line l, voxel i reads box par(kw) = (kw == 1), chunk (kd HR + 2 l + kh) 9 +
// i + (kw == 2): lines 18 chunks apart, channel groups 2 kBlk chunks apart.
template <int CI, int CO, int HR>
struct FpFwd {
  static constexpr int kC8 = CI / 8;
  static constexpr int kBlk = (3 * HR * 9 + 7) / 8 * 8;
  // HR = 17: lines 8..15 read past the loaded rows (garbage accumulator rows, never
  // stored); the last box's reads end (2 HR + 32) 9 + 9 chunks into it
  static constexpr int kTail = (2 * HR + 32) * 9 + 9 > kBlk ? (2 * HR + 32) * 9 + 9 - kBlk : 0;
  static constexpr int kFpBytes = (2 * kC8 * kBlk + (kTail + 7) / 8 * 8) * 16;
  static constexpr int kBoxBytes = 8 * 9 * HR * 3 * 2;  // bytes one box writes
  static constexpr int kWBytes = FpWeights<CI, CO>::kBytes;
  static constexpr int kSmem = 128 + kWBytes + kFpBytes + 64;  // + base alignment
  static constexpr uint32_t kLbo = 2 * kBlk * 16;  // channel group -> next
  static constexpr uint32_t kSbo = 18 * 16;        // line -> next (two input rows)
  static_assert(kSmem <= 227 * 1024, "footprint tile above the shared-memory limit");
};

template <int CI, int HR>
__device__ __forceinline__ void fp_fwd_tma(const CUtensorMap* xmap, const ConvShape& s, int t,
                                           uint8_t* fp, uint64_t* bar, int& b, int& od,
                                           int& oh0, int& ow0) {
  constexpr int kBlk = (3 * HR * 9 + 7) / 8 * 8;
  const int nwb = (s.Wo + 7) >> 3, nhb = (s.Ho + 15) >> 4;
  ow0 = (t % nwb) * 8;
  t /= nwb;
  oh0 = (t % nhb) * 16;
  t /= nhb;
  od = t % s.Do;
  b = t / s.Do;
#pragma unroll
  for (int c8 = 0; c8 < CI / 8; ++c8)
#pragma unroll
    for (int par = 0; par < 2; ++par)
      tma_load_5d(fp + (c8 * 2 + par) * kBlk * 16, xmap, c8 * 8, 2 * ow0 - 1 + par,
                  2 * oh0 - 1, 2 * od - 1, b, bar);
}

// Forward: pre = conv(x, w) + bias (FP32), act = GELU(pre) (BF16).  Persistent
// blocks: thread 0 loads the weight image once and each tile's footprint with TMA
// (bar[0]), issues the 27 taps' MMAs (bar[1]), and once they are done the next
// tile's footprint is requested before the epilogue reads this tile's accumulator.
template <int CI, int CO, int HR>
__global__ void __launch_bounds__(kFpThreads) k_conv_fp_fwd(const __grid_constant__ CUtensorMap xmap,
                                                            const __grid_constant__ CUtensorMap wmap,
                                                            ConvShape s, FwdEp ep, int* err) {
  using F = FpFwd<CI, CO, HR>;
  extern __shared__ __align__(128) uint8_t smem_raw[];
  uint8_t* const smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  uint8_t* const wimg = smem;
  uint8_t* const fp = smem + F::kWBytes;
  uint64_t* const bar = (uint64_t*)(fp + F::kFpBytes);  // [0] loads, [1] MMAs
  uint32_t* const slot = (uint32_t*)(bar + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntiles = s.B * s.Do * ((s.Ho + 15) >> 4) * ((s.Wo + 7) >> 3);

  int b = 0, od = 0, oh0 = 0, ow0 = 0;
  int t = blockIdx.x;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
    if (t < ntiles) {
      mbar_expect_tx(&bar[0], F::kWBytes + 2 * F::kC8 * F::kBoxBytes);
      fp_tma_weights<CI, CO>(wimg, &wmap, &bar[0]);
      fp_fwd_tma<CI, HR>(&xmap, s, t, fp, &bar[0], b, od, oh0, ow0);
    }
  }
  if (threadIdx.x != 0 && t < ntiles) {  // the tile coordinates, without issuing
    const int nwb = (s.Wo + 7) >> 3, nhb = (s.Ho + 15) >> 4;
    int u = t;
    ow0 = (u % nwb) * 8;
    u /= nwb;
    oh0 = (u % nhb) * 16;
    u /= nhb;
    od = u % s.Do;
    b = u / s.Do;
  }
  if (warp == 0) tc::tmem_alloc(slot, tc::tmem_cols<CO>());
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *slot;
  bool ok = true;
  int lost = -1;  // thread 0: a load wait that gave up (its copies may still land)
  for (int it = 0; t < ntiles; ++it) {
    bool lok = true;
    if (threadIdx.x == 0) {
      // the tile's footprint (and, first, the weights) have landed
      lok = mbar_wait_sleep_bounded(&bar[0], (uint32_t)(it & 1), err);
      if (!lok) lost = it;
      if (lok) {
        tc::fence_after_sync();
        const uint32_t wb = smem_u32(wimg), fb = smem_u32(fp);
        constexpr uint32_t idesc = tc::idesc_bf16_f32<128, CO>() | (1u << 16);  // B MN-major
        int n = 0;
#pragma unroll 1
        for (int tap = 0; tap < 27; ++tap) {
          const int kd = tap / 9, kh = (tap / 3) % 3, kw = tap % 3;
          const int aoff = (kw == 1 ? F::kBlk : 0) + (kd * HR + kh) * 9 + (kw == 2 ? 1 : 0);
#pragma unroll
          for (int kk = 0; kk < CI / 16; ++kk) {
            const uint32_t a = fb + (uint32_t)(aoff + 2 * kk * 2 * F::kBlk) * 16;
            const uint32_t bb = wb + (uint32_t)(tap * CI + 16 * kk) * 16;
            // B MN-major: K groups (8 ci) 128 bytes apart, N groups (8 co) 27 CI chunks
            tc::mma_bf16(tmem, fp_desc(a, F::kLbo, F::kSbo), fp_desc(bb, 128, 27 * CI * 16),
                         idesc, n++ > 0);
          }
        }
      }
      tc::commit(&bar[1]);  // also without MMAs, so the phase completes
    }
    ok = mbar_wait_block(&bar[1], (uint32_t)(it & 1), err, lok) && ok;
    tc::fence_after_sync();
    const int cb = b, cod = od, coh0 = oh0, cow0 = ow0;
    t += gridDim.x;
    if (!ok) break;
    if (t < ntiles) {  // the MMAs reading fp are done: request the next footprint
      if (threadIdx.x == 0) {
        mbar_expect_tx(&bar[0], 2 * F::kC8 * F::kBoxBytes);
        fp_fwd_tma<CI, HR>(&xmap, s, t, fp, &bar[0], b, od, oh0, ow0);
      } else {
        const int nwb = (s.Wo + 7) >> 3, nhb = (s.Ho + 15) >> 4;
        int u = t;
        ow0 = (u % nwb) * 8;
        u /= nwb;
        oh0 = (u % nhb) * 16;
        u /= nhb;
        od = u % s.Do;
        b = u / s.Do;
      }
    }
    const int q = warp & 3, row = q * 32 + lane;
    const int oh = coh0 + (row >> 3), ow = cow0 + (row & 7);
    const bool live = oh < s.Ho && ow < s.Wo;
    const int64_t m = (((int64_t)cb * s.Do + cod) * s.Ho + oh) * s.Wo + ow;
#pragma unroll
    for (int c = (warp >> 2) * (CO / 2); c < (warp >> 2 ? CO : CO / 2); c += 16) {
      float v[16];
      tc::ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c, v);
      if (live) ep.put16(m, c, 0, v);
    }
  }
  // copies whose wait gave up: one more bounded wait, so none lands after the block
  // has left
  if (threadIdx.x == 0 && lost >= 0) mbar_wait_sleep_bounded(&bar[0], (uint32_t)(lost & 1), err);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, tc::tmem_cols<CO>());
  }
}

// Data-gradient footprint (TMA): box co8 = dP[b, jd + dd, jh0 + hh, jw0 + ww,
// 8 co8 .. + 7], dd < 2, hh < 17, ww < 9, chunk (dd * 17 + hh) * 9 + ww, boxes 312
// chunks apart (128-byte aligned).
template <int CI, int CO>
struct FpDgrad {
  static constexpr int kBlk = 312;
  static constexpr int kBoxBytes = 8 * 9 * 17 * 2 * 2;
  static constexpr int kFpBytes = (CO / 8) * kBlk * 16;
  static constexpr int kWBytes = FpWeights<CI, CO>::kBytes;
  static constexpr int kSmem = 128 + kWBytes + kFpBytes + 64;
  static constexpr int kCols = 8 * CI;                // one accumulator per parity class
  static constexpr uint32_t kLbo = kBlk * 16;         // channel group -> next
  static constexpr uint32_t kSbo = 9 * 16;            // line -> next
  static_assert(kCols == 128 || kCols == 256 || kCols == 512, "TMEM allocation");
  static_assert(kSmem <= 227 * 1024, "footprint tile above the shared-memory limit");
};

// Tile t of the data gradient: (b, jd, jh0, jw0), and (thread 0) its dP boxes.
template <int CO>
__device__ __forceinline__ void fp_dgrad_tile(const CUtensorMap* dmap, const ConvShape& s, int t,
                                              uint8_t* fp, uint64_t* bar, bool issue,
                                              uint32_t extra_tx, int& b, int& jd, int& jh0,
                                              int& jw0) {
  const int nd = (s.D + 1) >> 1, nh = (s.H + 1) >> 1, nw = (s.W + 1) >> 1;
  const int nwb = (nw + 7) >> 3, nhb = (nh + 15) >> 4;
  jw0 = (t % nwb) * 8;
  t /= nwb;
  jh0 = (t % nhb) * 16;
  t /= nhb;
  jd = t % nd;
  b = t / nd;
  if (!issue) return;
  // one arrival per phase: the expected bytes of everything in flight on bar
  mbar_expect_tx(bar, extra_tx + (CO / 8) * FpDgrad<16, CO>::kBoxBytes);
#pragma unroll
  for (int co8 = 0; co8 < CO / 8; ++co8)
    tma_load_5d(fp + co8 * 312 * 16, dmap, co8 * 8, jw0, jh0, jd, b, bar);
}

// Data gradient of all eight parity classes of a tile of input voxels: dX[q, ci] =
// sum over the class's taps of dP[output reached through the tap] W[tap, ci, :].
// dx (FP32) or dxb (BF16) receives it.  Persistent blocks, loads and MMAs as in the
// forward.
template <int CI, int CO>
__global__ void __launch_bounds__(kFpThreads) k_conv_fp_dgrad(const __grid_constant__ CUtensorMap dmap,
                                                              const __grid_constant__ CUtensorMap wmap,
                                                              ConvShape s, float* __restrict__ dx,
                                                              bf16* __restrict__ dxb, int* err) {
  using F = FpDgrad<CI, CO>;
  extern __shared__ __align__(128) uint8_t smem_raw[];
  uint8_t* const smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  uint8_t* const wimg = smem;
  uint8_t* const fp = smem + F::kWBytes;
  uint64_t* const bar = (uint64_t*)(fp + F::kFpBytes);  // [0] loads, [1] MMAs
  uint32_t* const slot = (uint32_t*)(bar + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nd = (s.D + 1) >> 1, nh = (s.H + 1) >> 1, nw = (s.W + 1) >> 1;
  const int ntiles = s.B * nd * ((nh + 15) >> 4) * ((nw + 7) >> 3);

  int b = 0, jd = 0, jh0 = 0, jw0 = 0;
  int t = blockIdx.x;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  if (t < ntiles) {
    // the weights' bytes ride on the first footprint's expect_tx
    fp_dgrad_tile<CO>(&dmap, s, t, fp, &bar[0], threadIdx.x == 0, F::kWBytes, b, jd, jh0, jw0);
    if (threadIdx.x == 0) fp_tma_weights<CI, CO>(wimg, &wmap, &bar[0]);
  }
  if (warp == 0) tc::tmem_alloc(slot, F::kCols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *slot;
  bool ok = true;
  int lost = -1;
  for (int it = 0; t < ntiles; ++it) {
    bool lok = true;
    if (threadIdx.x == 0) {
      lok = mbar_wait_sleep_bounded(&bar[0], (uint32_t)(it & 1), err);
      if (!lok) lost = it;
      if (lok) {
        tc::fence_after_sync();
        const uint32_t wb = smem_u32(wimg), fb = smem_u32(fp);
        constexpr uint32_t idesc = tc::idesc_bf16_f32<128, CI>();  // both K-major
#pragma unroll 1
        for (int tap = 0; tap < 27; ++tap) {
          const int k[3] = {tap / 9, (tap / 3) % 3, tap % 3};
          // parity of the input voxels this tap reaches (k = 1: even; 0, 2: odd) and
          // the output offset (k = 0: j + 1, else j)
          int cls = 0, dl[3];
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            cls = cls * 2 + (k[a] == 1 ? 0 : 1);
            dl[a] = k[a] == 0 ? 1 : 0;
          }
          const int first = (k[0] != 2) && (k[1] != 2) && (k[2] != 2);  // first tap of its class
          const int aoff = (dl[0] * 17 + dl[1]) * 9 + dl[2];
#pragma unroll
          for (int kk = 0; kk < CO / 16; ++kk) {
            const uint32_t a = fb + (uint32_t)(aoff + 2 * kk * F::kBlk) * 16;
            const uint32_t bb = wb + (uint32_t)((2 * kk * 27 + tap) * CI) * 16;
            // B K-major: K groups (8 co) 27 CI chunks apart, N groups (8 ci) 128 bytes
            tc::mma_bf16(tmem + (uint32_t)(cls * CI), fp_desc(a, F::kLbo, F::kSbo),
                         fp_desc(bb, 27 * CI * 16, 128), idesc, !(first && kk == 0));
          }
        }
      }
      tc::commit(&bar[1]);  // also without MMAs, so the phase completes
    }
    ok = mbar_wait_block(&bar[1], (uint32_t)(it & 1), err, lok) && ok;
    tc::fence_after_sync();
    const int cb = b, cjd = jd, cjh0 = jh0, cjw0 = jw0;
    t += gridDim.x;
    if (!ok) break;
    if (t < ntiles)
      fp_dgrad_tile<CO>(&dmap, s, t, fp, &bar[0], threadIdx.x == 0, 0u, b, jd, jh0, jw0);
    const int q = warp & 3, row = q * 32 + lane;
    const int jh = cjh0 + (row >> 3), jw = cjw0 + (row & 7);
#pragma unroll 1
    for (int cls = (warp >> 2) * 4; cls < (warp >> 2) * 4 + 4; ++cls) {
      const int d = 2 * cjd + (cls >> 2), h = 2 * jh + ((cls >> 1) & 1), xw = 2 * jw + (cls & 1);
      const bool live = d < s.D && h < s.H && xw < s.W;
      const int64_t at = ((((int64_t)cb * s.D + d) * s.H + h) * s.W + xw) * CI;
#pragma unroll
      for (int c = 0; c < CI; c += 16) {
        float v[16];
        tc::ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(cls * CI + c), v);
        if (!live) continue;
        if (dxb) {
#pragma unroll
          for (int q8 = 0; q8 < 2; ++q8) {
            uint32_t u[4];
#pragma unroll
            for (int j = 0; j < 4; ++j)
              u[j] = pack2(__float2bfloat16(v[8 * q8 + 2 * j]),
                           __float2bfloat16(v[8 * q8 + 2 * j + 1]));
            *(uint4*)(dxb + at + c + 8 * q8) = make_uint4(u[0], u[1], u[2], u[3]);
          }
        } else {
#pragma unroll
          for (int q4 = 0; q4 < 4; ++q4)
            *(float4*)(dx + at + c + 4 * q4) =
                make_float4(v[4 * q4], v[4 * q4 + 1], v[4 * q4 + 2], v[4 * q4 + 3]);
        }
      }
    }
  }
  if (threadIdx.x == 0 && lost >= 0) mbar_wait_sleep_bounded(&bar[0], (uint32_t)(lost & 1), err);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, F::kCols);
  }
}

template <int CI, int CO>
struct FpWgrad {
  static constexpr int kC8 = CI / 8;
  static constexpr int kLoadRows = 33;
  // rows read: the last K step's second line starts at row 30; accumulator row
  // groups reach 16 / C8 - 1 rows further
  static constexpr int kPlaneRows = 30 + 16 / kC8;
  static constexpr int kPlaneChunks = kPlaneRows * kC8 * 18;
  static constexpr int kLoadChunks = kLoadRows * kC8 * 18;
  static constexpr int kDpChunks = (CO / 8) * 128;
  static constexpr int kStageBytes = (kPlaneChunks + kDpChunks) * 16;
  static constexpr int kOnesBytes = 512;
  static constexpr int kSmem = 2 * kStageBytes + kOnesBytes + 64;
  static constexpr int kCols = 4 * CO;  // kw = 0, 1, 2 and the bias
  static constexpr uint32_t kASbo = 18 * 16, kALbo = 36 * kC8 * 16;
  static constexpr uint32_t kBSbo = 128 * 16, kBLbo = 8 * 16;
  static_assert(kCols == 128 || kCols == 256, "TMEM allocation");
  static_assert(kSmem <= 227 * 1024, "footprint tile above the shared-memory limit");
};

// Plane kd of the forward footprint of tile t and its dP tile, into one stage.
template <int CI, int CO>
__device__ __forceinline__ void fp_wgrad_tile(const bf16* __restrict__ x,
                                              const bf16* __restrict__ dp, const ConvShape& s,
                                              int64_t t, int kd, uint8_t* plane, uint8_t* dps) {
  using F = FpWgrad<CI, CO>;
  const int nwb = (s.Wo + 7) >> 3, nhb = (s.Ho + 15) >> 4;
  const int owb = (int)(t % nwb);
  t /= nwb;
  const int ohb = (int)(t % nhb);
  t /= nhb;
  const int od = (int)(t % s.Do), b = (int)(t / s.Do);
  const int ow0 = owb * 8, oh0 = ohb * 16;
  const int d = 2 * od - 1 + kd, h0 = 2 * oh0 - 1, w0 = 2 * ow0 - 1;
  const bool dok = d >= 0 && d < s.D;
  // both in global order (coalesced full sectors), scattered into the layouts
  for (int e = threadIdx.x; e < F::kLoadChunks; e += kFpThreads) {
    const int c8 = e % F::kC8, q = e / F::kC8;
    const int wl = q % 18, hr = q / 18;
    const int h = h0 + hr, ww = w0 + wl;
    const bool in = dok && h >= 0 && h < s.H && ww >= 0 && ww < s.W;
    const bf16* src = in ? x + ((((size_t)b * s.D + d) * s.H + h) * s.W + ww) * CI + c8 * 8 : x;
    cp_async16(plane + (((hr * F::kC8 + c8) * 2 + (wl & 1)) * 9 + (wl >> 1)) * 16, src,
               in ? 16u : 0u);
  }
  for (int e = threadIdx.x; e < F::kDpChunks; e += kFpThreads) {
    const int co8 = e % (CO / 8), ml = e / (CO / 8);
    const int oh = oh0 + (ml >> 3), ow = ow0 + (ml & 7);
    const bool in = oh < s.Ho && ow < s.Wo;
    const bf16* src =
        in ? dp + ((((size_t)b * s.Do + od) * s.Ho + oh) * s.Wo + ow) * CO + co8 * 8 : dp;
    cp_async16(dps + (co8 * 128 + ml) * 16, src, in ? 16u : 0u);
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

// Weight and bias gradient partials: part[split][k][co] for k = tap * CI + ci of the
// block's plane kd (rows 27 CI .. Kp - 1 zero from block kd = 2, row Kp = db from
// block kd = 1); split = blockIdx.x takes forward tiles [split * per, ..).  Two
// stages: tile it + 1 is copied while the MMAs of tile it run.
template <int CI, int CO>
__global__ void __launch_bounds__(kFpThreads) k_conv_fp_wgrad(const bf16* __restrict__ x,
                                                              ConvShape s,
                                                              const bf16* __restrict__ dp,
                                                              int per, float* __restrict__ part,
                                                              int* err) {
  using F = FpWgrad<CI, CO>;
  extern __shared__ __align__(128) uint8_t smem[];
  uint8_t* const ones = smem + 2 * F::kStageBytes;
  uint64_t* const bar = (uint64_t*)(ones + F::kOnesBytes);
  uint32_t* const slot = (uint32_t*)(bar + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kd = blockIdx.y;
  const int64_t ntiles = (int64_t)s.B * s.Do * ((s.Ho + 15) >> 4) * ((s.Wo + 7) >> 3);
  const int64_t t0 = (int64_t)blockIdx.x * per;
  const int64_t left = ntiles - t0;
  const int nt = left <= 0 ? 0 : (int)(left < per ? left : per);

  for (int e = threadIdx.x; e < F::kOnesBytes / 4; e += kFpThreads)
    ((uint32_t*)ones)[e] = 0x3F803F80u;
  if (nt > 0) fp_wgrad_tile<CI, CO>(x, dp, s, t0, kd, smem, smem + F::kPlaneChunks * 16);
  if (warp == 0) tc::tmem_alloc(slot, F::kCols);
  if (threadIdx.x == 32) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *slot;

  bool ok = true;
  int issued = 0;
  for (int it = 0; it < nt; ++it) {
    const int st = it & 1;
    uint8_t* const plane = smem + st * F::kStageBytes;
    uint8_t* const dps = plane + F::kPlaneChunks * 16;
    if (it + 1 < nt) {
      // stage (it + 1) & 1 was read by the MMAs of tile it - 1: wait for their commit
      if (it >= 1) ok = mbar_wait_bounded(&bar[st ^ 1], (uint32_t)(((it - 1) >> 1) & 1), err) && ok;
      uint8_t* const nplane = smem + (st ^ 1) * F::kStageBytes;
      fp_wgrad_tile<CI, CO>(x, dp, s, t0 + it + 1, kd, nplane, nplane + F::kPlaneChunks * 16);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    fence_proxy_async();
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    if (threadIdx.x == 0) {
      tc::fence_after_sync();
      const uint32_t pa = smem_u32(plane), pb = smem_u32(dps), po = smem_u32(ones);
      constexpr uint32_t idesc = tc::idesc_bf16_f32<128, CO>() | (1u << 15) | (1u << 16);
#pragma unroll 1
      for (int q = 0; q < 8; ++q) {  // lines 2q, 2q + 1
        const uint32_t bq = pb + (uint32_t)(16 * q) * 16;
        const uint64_t bdesc = fp_desc(bq, F::kBLbo, F::kBSbo);
#pragma unroll
        for (int kw = 0; kw < 3; ++kw) {
          const int aoff = 4 * q * F::kC8 * 18 + (kw == 1 ? 9 : 0) + (kw == 2 ? 1 : 0);
          tc::mma_bf16(tmem + (uint32_t)(kw * CO),
                       fp_desc(pa + (uint32_t)aoff * 16, F::kALbo, F::kASbo), bdesc, idesc,
                       it > 0 || q > 0);
        }
        if (kd == 1)  // A = ones: every accumulator row is sum_m dP[m, co]
          tc::mma_bf16(tmem + (uint32_t)(3 * CO), fp_desc(po, 128, 16), bdesc, idesc,
                       it > 0 || q > 0);
      }
      tc::commit(&bar[st]);
    }
    issued = it + 1;
  }
  cp_async_wait_all();  // copies of a tile the loop left early
  // the last two commits: every MMA of the block is done, and no commit arrives on a
  // barrier after the block has left
  for (int it = issued >= 2 ? issued - 2 : 0; it < issued; ++it)
    ok = mbar_wait_bounded(&bar[it & 1], (uint32_t)((it >> 1) & 1), err) && ok;
  tc::fence_after_sync();

  float* const pw = part + (int64_t)blockIdx.x * (s.Kp + 1) * CO;
  const int q = warp & 3, row = q * 32 + lane, c0 = (warp >> 2) * (CO / 2);
  const int g = row >> 3, kh = g / F::kC8, ci = (g % F::kC8) * 8 + (row & 7);
  const bool live = ok && issued > 0 && kh < 3;
#pragma unroll 1
  for (int kw = 0; kw < 3; ++kw) {
    float* const dst = pw + (int64_t)(((kd * 3 + kh) * 3 + kw) * CI + ci) * CO;
#pragma unroll
    for (int c = c0; c < c0 + CO / 2; c += 16) {
      float v[16];
      tc::ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(kw * CO + c), v);
      if (!live) continue;
#pragma unroll
      for (int q4 = 0; q4 < 4; ++q4)
        *(float4*)(dst + c + 4 * q4) =
            make_float4(v[4 * q4], v[4 * q4 + 1], v[4 * q4 + 2], v[4 * q4 + 3]);
    }
  }
  if (kd == 1 && q == 0) {
#pragma unroll
    for (int c = c0; c < c0 + CO / 2; c += 16) {
      float v[16];
      tc::ld16(tmem + (uint32_t)(3 * CO + c), v);
      if (lane == 0 && ok && issued > 0)
#pragma unroll
        for (int j = 0; j < 16; ++j) pw[(int64_t)s.Kp * CO + c + j] = v[j];
    }
  }
  if (kd == 2)  // padding rows of W
    for (int i = threadIdx.x; i < (s.Kp - 27 * CI) * CO; i += kFpThreads) pw[27 * CI * CO + i] = 0.f;
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, F::kCols);
  }
}

}  // namespace dm
