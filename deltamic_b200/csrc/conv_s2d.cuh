// Single-channel layer (Ci = 1, the encoder's first) on the tensor cores, as a
// space-to-depth convolution (included by conv.cu after conv_fp.cuh).
//
// Input block (bd, bh, bw) holds the 2 x 2 x 2 voxels x[b, 2 bd + pd, 2 bh + ph,
// 2 bw + pw] as eight BF16 channels par = 4 pd + 2 ph + pw: one 16-byte chunk.  Tap k
// of an axis reads input 2 o - 1 + k, i.e. block o - 1 (parity 1) for k = 0 and block
// o (parity 0, 1) for k = 1, 2; so the stride-2 3x3x3 convolution is a stride-1
// 2 x 2 x 2 convolution over blocks (o - 1 + dd, o - 1 + dh, o - 1 + dw), dd, dh,
// dw in {0, 1}, with 8 channels per block and 27 of the 64 weights per output
// channel non-zero ((dd, p) = (0, 0) reaches no tap).
//
// A tile is 16 output lines x 8 voxels (128 rows).  Its block footprint is
// chunk ((dd * 17 + hh) * 9 + ww) for blocks (od - 1 + dd, oh0 - 1 + hh, ow0 - 1 + ww)
// (zero outside the volume), each block's four (pd, ph) column pairs 4 bytes apart:
// the forward stages it through registers from aligned 16-byte row pieces, the
// weight gradient with 4-byte cp.async copies.  8 consecutive voxels of a line are 8 consecutive chunks, and
// the block tap dw is one chunk further: the forward's A operand (K-major, K = (dw,
// par)) is the footprint itself with a leading byte offset of 16 (the two core
// matrices along K overlap by seven rows) and lines 9 chunks apart.  Four MMAs, one
// per (dd, dh), make a tile.
//
// The weight gradient reads the same footprint as the MN-major A operand of
// dW^T[(block tap, par), co] = sum_m X[m + tap][par] dP[m, co], with the eight block
// taps expanded into 2-KB groups of 128 chunks (group 8: ones, the bias row).
#pragma once

namespace dm {

__device__ __forceinline__ void cp_async4(void* dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}

constexpr int kS2dFpChunks = 2 * 17 * 9;  // block footprint of a tile
constexpr int kS2dFpBytes = 4992;         // 306 chunks, padded to 128 bytes

// Tap of block tap (dd, dh, dw) and parity par (4 pd + 2 ph + pw), or -1.
__device__ __forceinline__ int s2d_tap(int btap, int par) {
  int tap = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int dl = (btap >> (2 - a)) & 1, p = (par >> (2 - a)) & 1;
    if (dl == 0 && p == 0) return -1;
    tap = tap * 3 + (dl == 0 ? 0 : 1 + p);
  }
  return tap;
}

// Block footprint of the tile of output lines (b, od, oh0 .. oh0 + 15), voxels
// ow0 .. ow0 + 7.  Lanes take consecutive blocks of a (pd, ph) input row (4-byte
// column pairs, coalesced); needs W even and x 4-byte aligned.
__device__ __forceinline__ void s2d_footprint(const bf16* __restrict__ x, const ConvShape& s,
                                              int b, int od, int oh0, int ow0, uint8_t* fp,
                                              int nthreads) {
  for (int e = threadIdx.x; e < kS2dFpChunks * 4; e += nthreads) {
    const int ww = e % 9, r = e / 9;
    const int pp = r & 3, r2 = r >> 2;
    const int hh = r2 % 17, dd = r2 / 17;
    const int d = 2 * (od - 1 + dd) + (pp >> 1), h = 2 * (oh0 - 1 + hh) + (pp & 1);
    const int w = 2 * (ow0 - 1 + ww);
    const bool ok = d >= 0 && d < s.D && h >= 0 && h < s.H && w >= 0 && w + 1 < s.W;
    const bf16* src = ok ? x + (((size_t)b * s.D + d) * s.H + h) * s.W + w : x;
    cp_async4(fp + ((dd * 17 + hh) * 9 + ww) * 16 + pp * 4, src, ok ? 4u : 0u);
  }
}

// The forward's footprint through registers: a (dd, hh, pp) input row segment of a
// tile spans columns 2 ow0 - 2 .. 2 ow0 + 15; it is read as the three aligned
// 16-byte pieces 2 ow0 - 8 + 8 j .. + 7 (needs W a multiple of 8 and x 16-byte
// aligned), whose column pairs t are blocks ww = 4 j + t - 3.  Loads are issued
// first (s2d_prefetch) and stored after the epilogue (s2d_store), so their latency
// hides behind it.  Thread items: e = threadIdx.x + 256 i, i < 2, of 408.
struct S2dPrefetch {
  uint4 v[2];
  int16_t dst[2];  // chunk * 4 + pp of the row segment; -1: no item
  int8_t j[2];
};

__device__ __forceinline__ void s2d_prefetch(const bf16* __restrict__ x, const ConvShape& s,
                                             int b, int od, int oh0, int ow0, S2dPrefetch& p) {
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int e = threadIdx.x + 256 * i;
    p.dst[i] = -1;
    p.v[i] = make_uint4(0u, 0u, 0u, 0u);
    if (e >= 136 * 3) continue;
    const int j = e % 3, rr = e / 3;
    const int pp = rr & 3, r2 = rr >> 2;
    const int hh = r2 % 17, dd = r2 / 17;
    const int d = 2 * (od - 1 + dd) + (pp >> 1), h = 2 * (oh0 - 1 + hh) + (pp & 1);
    const int c0 = 2 * ow0 - 8 + 8 * j;
    p.dst[i] = (int16_t)(((dd * 17 + hh) * 9) * 4 + pp);
    p.j[i] = (int8_t)j;
    if (d < 0 || d >= s.D || h < 0 || h >= s.H) continue;
    const bf16* row = x + (((size_t)b * s.D + d) * s.H + h) * s.W;
    if (c0 >= 0 && c0 + 8 <= s.W) {
      p.v[i] = __ldg((const uint4*)(row + c0));
    } else {  // a piece at the volume's edge
      uint16_t e8[8];
#pragma unroll
      for (int k = 0; k < 8; ++k)
        e8[k] = (c0 + k >= 0 && c0 + k < s.W) ? __bfloat16_as_ushort(row[c0 + k]) : (uint16_t)0;
      p.v[i] = make_uint4(e8[0] | (uint32_t)e8[1] << 16, e8[2] | (uint32_t)e8[3] << 16,
                          e8[4] | (uint32_t)e8[5] << 16, e8[6] | (uint32_t)e8[7] << 16);
    }
  }
}

__device__ __forceinline__ void s2d_store(uint8_t* fp, const S2dPrefetch& p) {
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    if (p.dst[i] < 0) continue;
    const int chunk4 = p.dst[i] >> 2, pp = p.dst[i] & 3, j = p.j[i];
    const uint32_t w4[4] = {p.v[i].x, p.v[i].y, p.v[i].z, p.v[i].w};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int ww = 4 * j + t - 3;
      if (ww >= 0 && ww < 9) *(uint32_t*)(fp + (chunk4 + ww) * 16 + pp * 4) = w4[t];
    }
  }
}

// The same for a group of 128 threads (t = its thread index): items t + 128 i, i < 4.
struct S2dPrefetch4 {
  uint4 v[4];
  int16_t dst[4];
  int8_t j[4];
};

__device__ __forceinline__ void s2d_prefetch4(const bf16* __restrict__ x, const ConvShape& s,
                                              int b, int od, int oh0, int ow0, int t,
                                              S2dPrefetch4& p) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int e = t + 128 * i;
    p.dst[i] = -1;
    p.v[i] = make_uint4(0u, 0u, 0u, 0u);
    if (e >= 136 * 3) continue;
    const int j = e % 3, rr = e / 3;
    const int pp = rr & 3, r2 = rr >> 2;
    const int hh = r2 % 17, dd = r2 / 17;
    const int d = 2 * (od - 1 + dd) + (pp >> 1), h = 2 * (oh0 - 1 + hh) + (pp & 1);
    const int c0 = 2 * ow0 - 8 + 8 * j;
    p.dst[i] = (int16_t)(((dd * 17 + hh) * 9) * 4 + pp);
    p.j[i] = (int8_t)j;
    if (d < 0 || d >= s.D || h < 0 || h >= s.H) continue;
    const bf16* row = x + (((size_t)b * s.D + d) * s.H + h) * s.W;
    if (c0 >= 0 && c0 + 8 <= s.W) {
      p.v[i] = __ldg((const uint4*)(row + c0));
    } else {  // a piece at the volume's edge
      uint16_t e8[8];
#pragma unroll
      for (int k = 0; k < 8; ++k)
        e8[k] = (c0 + k >= 0 && c0 + k < s.W) ? __bfloat16_as_ushort(row[c0 + k]) : (uint16_t)0;
      p.v[i] = make_uint4(e8[0] | (uint32_t)e8[1] << 16, e8[2] | (uint32_t)e8[3] << 16,
                          e8[4] | (uint32_t)e8[5] << 16, e8[6] | (uint32_t)e8[7] << 16);
    }
  }
}

__device__ __forceinline__ void s2d_store4(uint8_t* fp, const S2dPrefetch4& p) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (p.dst[i] < 0) continue;
    const int chunk4 = p.dst[i] >> 2, pp = p.dst[i] & 3, j = p.j[i];
    const uint32_t w4[4] = {p.v[i].x, p.v[i].y, p.v[i].z, p.v[i].w};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int ww = 4 * j + t - 3;
      if (ww >= 0 && ww < 9) *(uint32_t*)(fp + (chunk4 + ww) * 16 + pp * 4) = w4[t];
    }
  }
}

// Warp-specialized forward of the single-channel layer.  Warps 4-7 stage a tile's
// block footprint (register loads of aligned row pieces, two footprint buffers) and
// one of their threads issues its four MMAs into one of two TMEM accumulators;
// warps 0-3 run the bias + GELU epilogue of the other accumulator meanwhile (one
// output row per thread, all CO channels).  Barriers: mdone[buffer] (the MMAs that
// read a footprint buffer are done), tfull / tempty[accumulator].
template <int CO>
struct S2dFwdWs {
  static constexpr int kWBytes = 8 * CO * 16;
  static constexpr int kSmem = kWBytes + 2 * kS2dFpBytes + 128;
  static constexpr int kCols = 2 * CO < 32 ? 32 : 2 * CO;
};

template <int CO>
__global__ void __launch_bounds__(256) k_conv_s2d_fwd_ws(const bf16* __restrict__ x, ConvShape s,
                                                         const bf16* __restrict__ w,
                                                         const float* __restrict__ bias,
                                                         float* __restrict__ pre,
                                                         bf16* __restrict__ act, int* err) {
  using F = S2dFwdWs<CO>;
  extern __shared__ __align__(128) uint8_t smem[];
  uint8_t* const wimg = smem;
  uint8_t* const fps = smem + F::kWBytes;
  uint64_t* const mdone = (uint64_t*)(fps + 2 * kS2dFpBytes);
  uint64_t* const tfull = mdone + 2;
  uint64_t* const tempty = tfull + 2;
  uint64_t* const done = tempty + 2;
  uint32_t* const slot = (uint32_t*)(done + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwb = (s.Wo + 7) >> 3, nhb = (s.Ho + 15) >> 4;
  const int ntiles = s.B * s.Do * nhb * nwb;
  const int nloc = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  auto tile = [&](int lt, int& b, int& od, int& oh0, int& ow0) {
    int t = (int)blockIdx.x + lt * (int)gridDim.x;
    ow0 = (t % nwb) * 8;
    t /= nwb;
    oh0 = (t % nhb) * 16;
    t /= nhb;
    od = t % s.Do;
    b = t / s.Do;
  };

  for (int e = threadIdx.x; e < 8 * CO * 8; e += 256) {  // weight image (K-major B)
    const int par = e & 7, co = (e >> 3) % CO, btap = (e >> 3) / CO;
    const int tap = s2d_tap(btap, par);
    ((bf16*)wimg)[e] = tap < 0 ? __float2bfloat16(0.f) : w[tap * CO + co];
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(&mdone[i], 1);
      mbar_init(&tfull[i], 1);
      mbar_init(&tempty[i], 4);
    }
    mbar_init(done, 1);
    fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(slot, F::kCols);
  fence_proxy_async();  // weight image -> the MMA's async-proxy reads
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *slot;

  if (warp >= 4) {  // producer
    const int t = threadIdx.x - 128;
    bool good = true;
    S2dPrefetch4 pf;  // the pieces of the tile about to be stored, loaded a tile ahead
    if (nloc > 0) {
      int b, od, oh0, ow0;
      tile(0, b, od, oh0, ow0);
      s2d_prefetch4(x, s, b, od, oh0, ow0, t, pf);
    }
    for (int lt = 0; lt < nloc && good; ++lt) {
      const int fb = lt & 1, acc = lt & 1;
      // the MMAs of tile lt - 2 read this footprint buffer
      if (lt >= 2 && !mbar_wait_sleep_bounded(&mdone[fb], (uint32_t)(((lt - 2) >> 1) & 1), err))
        good = false;
      if (good) s2d_store4(fps + fb * kS2dFpBytes, pf);
      fence_proxy_async();
      good = named_bar_and(1, 128, good);  // the footprint is stored, by every producer
      if (!good) break;
      if (lt + 1 < nloc) {  // next tile's loads in flight while this tile's MMAs issue
        int b, od, oh0, ow0;
        tile(lt + 1, b, od, oh0, ow0);
        s2d_prefetch4(x, s, b, od, oh0, ow0, t, pf);
      }
      if (t == 0) {
        if (lt >= 2 &&
            !mbar_wait_sleep_bounded(&tempty[acc], (uint32_t)(((lt >> 1) - 1) & 1), err)) {
          good = false;
        } else {
          tc::fence_after_sync();
          const uint32_t wb = smem_u32(wimg), fb0 = smem_u32(fps + fb * kS2dFpBytes);
          constexpr uint32_t idesc = tc::idesc_bf16_f32<128, CO>();  // both K-major
#pragma unroll
          for (int g = 0; g < 4; ++g) {  // (dd, dh); K = (dw, par)
            const uint32_t a = fb0 + (uint32_t)(((g >> 1) * 17 + (g & 1)) * 9) * 16;
            const uint32_t bb = wb + (uint32_t)(2 * g * CO) * 16;
            tc::mma_bf16(tmem + (uint32_t)(acc * CO), fp_desc(a, 16, 9 * 16),
                         fp_desc(bb, CO * 16, 128), idesc, g > 0);
          }
        }
        tc::commit(&mdone[fb]);
        tc::commit(&tfull[acc]);
      }
      good = named_bar_and(1, 128, good);  // thread 0's accumulator wait, shared
    }
    if (t == 0) {  // every MMA issued is complete before the block leaves
      tc::commit(done);
      mbar_wait_sleep_bounded(done, 0u, err);
    }
  } else {  // epilogue: warp q reads TMEM lane quarter q
    const int row = warp * 32 + lane;
    float bv[CO];
#pragma unroll
    for (int j = 0; j < CO; ++j) bv[j] = bias ? bias[j] : 0.f;
    for (int lt = 0; lt < nloc; ++lt) {
      const int acc = lt & 1;
      int ok = 1;
      if (lane == 0) ok = mbar_wait_sleep_bounded(&tfull[acc], (uint32_t)((lt >> 1) & 1), err);
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      if (lane != 0) mbar_wait_bounded(&tfull[acc], (uint32_t)((lt >> 1) & 1), err);
      tc::fence_after_sync();
      int b, od, oh0, ow0;
      tile(lt, b, od, oh0, ow0);
      const int oh = oh0 + (row >> 3), ow = ow0 + (row & 7);
      const bool live = oh < s.Ho && ow < s.Wo;
      const int64_t m = (((int64_t)b * s.Do + od) * s.Ho + oh) * s.Wo + ow;
#pragma unroll
      for (int c = 0; c < CO; c += 16) {
        float v[16];
        tc::ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(acc * CO + c), v);
        if (!live) continue;
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] += bv[c + j];
        float4* pp = (float4*)(pre + m * CO + c);
#pragma unroll
        for (int q = 0; q < 4; ++q) pp[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        uint32_t u[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
          u[j] = pack2(__float2bfloat16(gelu(v[2 * j])), __float2bfloat16(gelu(v[2 * j + 1])));
        *(uint4*)(act + m * CO + c) = make_uint4(u[0], u[1], u[2], u[3]);
        *(uint4*)(act + m * CO + c + 8) = make_uint4(u[4], u[5], u[6], u[7]);
      }
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive1(&tempty[acc]);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, F::kCols);
  }
}

template <int CO>
struct S2dWgrad {
  static constexpr int kGroupBytes = 128 * 16;       // one block tap's 128 voxels
  static constexpr int kABytes = 9 * kGroupBytes;     // groups 0..7 taps, 8 ones
  // accumulator rows of groups 9..15 are never stored; their reads run on into the
  // next stage's region and this pad
  static constexpr int kARegion = 2 * kABytes + 7 * kGroupBytes;
  static constexpr int kDpBytes = (CO / 8) * 128 * 16;
  static constexpr int kSmem = kARegion + 2 * kS2dFpBytes + 2 * kDpBytes + 64;
};

// Weight + bias gradient partials of the single-channel layer: split = blockIdx.x
// sums tiles [split * per, ..) into part[split][k][co] (k = tap, rows 27 .. Kp - 1
// zero, row Kp = db).  Per tile: the block footprint and dP tile are copied one tile
// ahead (two stages), the footprint is expanded into the eight block-tap groups, and
// eight MMAs (M = 128: group x parity, N = CO, K = 16 voxels) accumulate in TMEM.
// VEC (W a multiple of 8, x 16-byte aligned): the footprint through registers as in
// the forward -- tile it + 1's pieces are loaded before tile it's expansion and
// stored after its MMAs are issued; else 4-byte cp.async copies.
template <int CO, bool VEC>
__global__ void __launch_bounds__(256) k_conv_s2d_wgrad(const bf16* __restrict__ x, ConvShape s,
                                                        const bf16* __restrict__ dp, int per,
                                                        float* __restrict__ part, int* err) {
  using F = S2dWgrad<CO>;
  extern __shared__ __align__(128) uint8_t smem[];
  uint8_t* const areg = smem;
  uint8_t* const fps = smem + F::kARegion;
  uint8_t* const dps = fps + 2 * kS2dFpBytes;
  uint64_t* const bar = (uint64_t*)(dps + 2 * F::kDpBytes);
  uint32_t* const slot = (uint32_t*)(bar + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwb = (s.Wo + 7) >> 3, nhb = (s.Ho + 15) >> 4;
  const int64_t ntiles = (int64_t)s.B * s.Do * nhb * nwb;
  const int64_t t0 = (int64_t)blockIdx.x * per;
  const int64_t left = ntiles - t0;
  const int nt = left <= 0 ? 0 : (int)(left < per ? left : per);

  // tile it's copies into stage st: block footprint (or, VEC, its pieces into pf) and
  // dP [co8][voxel]
  S2dPrefetch pf;
  auto load = [&](int it, int st) {
    int64_t t = t0 + it;
    const int ow0 = (int)(t % nwb) * 8;
    t /= nwb;
    const int oh0 = (int)(t % nhb) * 16;
    t /= nhb;
    const int od = (int)(t % s.Do), b = (int)(t / s.Do);
    if (VEC)
      s2d_prefetch(x, s, b, od, oh0, ow0, pf);
    else
      s2d_footprint(x, s, b, od, oh0, ow0, fps + st * kS2dFpBytes, 256);
    uint8_t* const d = dps + st * F::kDpBytes;
    for (int e = threadIdx.x; e < (CO / 8) * 128; e += 256) {
      const int co8 = e % (CO / 8), ml = e / (CO / 8);
      const int oh = oh0 + (ml >> 3), ow = ow0 + (ml & 7);
      const bool in = oh < s.Ho && ow < s.Wo;
      const bf16* src =
          in ? dp + ((((size_t)b * s.Do + od) * s.Ho + oh) * s.Wo + ow) * CO + co8 * 8 : dp;
      cp_async16(d + (co8 * 128 + ml) * 16, src, in ? 16u : 0u);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };

  for (int e = threadIdx.x; e < 2 * F::kGroupBytes / 4; e += 256) {  // the ones groups
    const int st = e / (F::kGroupBytes / 4), o = e % (F::kGroupBytes / 4);
    ((uint32_t*)(areg + st * F::kABytes + 8 * F::kGroupBytes))[o] = 0x3F803F80u;
  }
  if (nt > 0) {
    load(0, 0);
    if (VEC) s2d_store(fps, pf);
  }
  if (warp == 0) tc::tmem_alloc(slot, 32);
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
    if (it + 1 < nt) {
      // stage st ^ 1 (dP and A) was read by the MMAs of tile it - 1
      if (it >= 1) ok = mbar_wait_bounded(&bar[st ^ 1], (uint32_t)(((it - 1) >> 1) & 1), err) && ok;
      load(it + 1, st ^ 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();  // tile it's footprint is complete
    // expand: group g = (dd, dh, dw), voxel (l, i) <- footprint block (dd, l + dh, i + dw)
    const uint8_t* const f = fps + st * kS2dFpBytes;
    uint8_t* const a = areg + st * F::kABytes;
    for (int e = threadIdx.x; e < 8 * 128; e += 256) {
      const int g = e >> 7, ml = e & 127;
      const int src = (((g >> 2) * 17 + (ml >> 3) + ((g >> 1) & 1)) * 9) + (ml & 7) + (g & 1);
      *(uint4*)(a + e * 16) = *(const uint4*)(f + src * 16);
    }
    fence_proxy_async();
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    if (threadIdx.x == 0) {
      tc::fence_after_sync();
      const uint32_t pa = smem_u32(a), pb = smem_u32(dps + st * F::kDpBytes);
      constexpr uint32_t idesc = tc::idesc_bf16_f32<128, CO>() | (1u << 15) | (1u << 16);
#pragma unroll
      for (int q = 0; q < 8; ++q)  // voxels 16 q .. 16 q + 15
        tc::mma_bf16(tmem, fp_desc(pa + q * 256, 128, F::kGroupBytes),
                     fp_desc(pb + q * 256, 128, 128 * 16), idesc, it > 0 || q > 0);
      tc::commit(&bar[st]);
    }
    issued = it + 1;
    // the next tile's pieces: its footprint stage was expanded an iteration ago
    if (VEC && it + 1 < nt) s2d_store(fps + (st ^ 1) * kS2dFpBytes, pf);
  }
  cp_async_wait_all();
  for (int it = issued >= 2 ? issued - 2 : 0; it < issued; ++it)
    ok = mbar_wait_bounded(&bar[it & 1], (uint32_t)((it >> 1) & 1), err) && ok;
  tc::fence_after_sync();

  float* const pw = part + (int64_t)blockIdx.x * (s.Kp + 1) * CO;
  const int q = warp & 3, row = q * 32 + lane, c0 = (warp >> 2) * (CO / 2);
  const int g = row >> 3, par = row & 7;
  const int tap = g < 8 ? s2d_tap(g, par) : -1;
  const bool live = ok && issued > 0;
  if (q < 3) {
#pragma unroll
    for (int c = 0; c < CO / 2; c += 8) {
      float v[8];
      tc::ld8(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(c0 + c), v);
      if (!live) continue;
      float* dst = tap >= 0 ? pw + (int64_t)tap * CO : (row == 64 ? pw + (int64_t)s.Kp * CO : nullptr);
      if (dst) {
        *(float4*)(dst + c0 + c) = make_float4(v[0], v[1], v[2], v[3]);
        *(float4*)(dst + c0 + c + 4) = make_float4(v[4], v[5], v[6], v[7]);
      }
    }
  }
  for (int i = threadIdx.x; i < (s.Kp - 27) * CO; i += 256) pw[27 * CO + i] = 0.f;
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, 32);
  }
}

}  // namespace dm
