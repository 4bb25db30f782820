// Tap-GEMM forward for layers with 64 input channels and few output voxels per
// image (the encoder's last layer, 64 -> 128 at 4^3 outputs), included by conv.cu.
//
// A tap's 64 input channels are one 128-byte row, so for tap (kd, kh, kw) the A tile
// of 128 output voxels (whole images: 128 / (Do Ho Wo) of them) is one TMA box of x
// with a traversal stride of 2 along W, H and D, starting at input (kw - 1, kh - 1,
// kd - 1): rows in output-voxel order, 64 channels each, written with the 128-byte
// swizzle -- the canonical K-major SW128 operand (8-row groups 1024 bytes apart,
// K = 16 steps 32 bytes further along the row).  The B tile is the tap's 64 rows of
// W, read MN-major (two boxes of 64 output channels; 8-row K groups 1024 bytes
// apart, a K = 16 step 2048 bytes).  The
// 27 taps are split over blockIdx.y; each block accumulates its taps in TMEM and
// writes FP32 partials part[split][m][co], added in split order with the bias and
// GELU by k_fwd_reduce.  No gathers: the TMA engine fetches the taps, one thread
// issues copies and MMAs through a ring of stages.
#pragma once

namespace dm {

constexpr int kTgStages = 3;
constexpr int kTgStageBytes = 2 * 128 * 128;  // A and B tiles, 128 rows x 128 bytes each

// SW128 K-major descriptor: start address, LBO 16 bytes (unused by this layout),
// SBO 1024 bytes (8-row groups), version 1, layout type 2 (128-byte swizzle).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) |
         ((uint64_t)(1024u >> 4) << 32) | (1ull << 46) | (2ull << 61);
}

// MN-major SW128 descriptor: 64-element MN groups ``lbo`` bytes apart, 8-row K
// groups 1024 bytes apart (a K = 16 step is 2048 bytes), layout type 2.
__device__ __forceinline__ uint64_t sw128_mn_desc(uint32_t saddr, uint32_t lbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)(1024u >> 4) << 32) | (1ull << 46) | (2ull << 61);
}

// Layout type of an R-byte row swizzle (R = 32, 64, 128).
__host__ __device__ constexpr uint32_t swz_code(int row_bytes) {
  return row_bytes == 32 ? 6u : (row_bytes == 64 ? 4u : 2u);
}
// Swizzled K-major descriptor for R-byte rows (8-row groups 8 R bytes apart).
template <int R>
__device__ __forceinline__ uint64_t swk_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) |
         ((uint64_t)((8 * R) >> 4) << 32) | (1ull << 46) | ((uint64_t)swz_code(R) << 61);
}
// Swizzled MN-major descriptor for R-byte rows: MN groups lbo bytes apart, 8-row K
// groups 8 R bytes apart.
template <int R>
__device__ __forceinline__ uint64_t swmn_desc(uint32_t saddr, uint32_t lbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((8 * R) >> 4) << 32) | (1ull << 46) | ((uint64_t)swz_code(R) << 61);
}

// Block (m tile, split): taps [split * tps, ..) of output rows [128 m, 128 m + 128).
// 128 threads: thread 0 issues, then all four warps read their TMEM lane quarter.
__global__ void __launch_bounds__(128) k_conv_tg_fwd(const __grid_constant__ CUtensorMap xmap,
                                                     const __grid_constant__ CUtensorMap wmap,
                                                     ConvShape s, int tps, float* __restrict__ part,
                                                     int* err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* const smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint64_t* const full = (uint64_t*)(smem + kTgStages * kTgStageBytes);
  uint64_t* const empty = full + kTgStages;
  uint64_t* const done = empty + kTgStages;
  uint32_t* const slot = (uint32_t*)(done + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int per_img = s.Do * s.Ho * s.Wo, nb = 128 / per_img;
  const int b0 = blockIdx.x * nb;
  const int t0 = blockIdx.y * tps, nt = min(27, t0 + tps) - t0;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kTgStages; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(done, 1);
    fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(slot, 128);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *slot;

  int lost = 0;  // thread 0: a wait gave up (copies may be in flight)
  if (threadIdx.x == 0) {
    auto load = [&](int i) {
      const int st = i % kTgStages, tap = t0 + i;
      const int kd = tap / 9, kh = (tap / 3) % 3, kw = tap % 3;
      uint8_t* a = smem + st * kTgStageBytes;
      mbar_expect_tx(&full[st], kTgStageBytes);
      tma_load_5d(a, &xmap, 0, kw - 1, kh - 1, kd - 1, b0, &full[st]);
#pragma unroll
      for (int h = 0; h < 2; ++h)  // W rows of the tap, 64 output channels per box
        tma_load_2d(a + 128 * 128 + h * 64 * 128, &wmap, 64 * h, tap * 64, &full[st]);
    };
    for (int i = 0; i < nt && i < kTgStages; ++i) load(i);
    constexpr uint32_t idesc = tc::idesc_bf16_f32<128, 128>() | (1u << 16);  // B MN-major
    for (int i = 0; i < nt; ++i) {
      const int st = i % kTgStages;
      if (!mbar_wait_sleep_bounded(&full[st], (uint32_t)((i / kTgStages) & 1), err)) {
        lost = 1;
        break;
      }
      tc::fence_after_sync();
      const uint32_t a = smem_u32(smem + st * kTgStageBytes), b = a + 128 * 128;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)  // K = 64 channels: four K = 16 steps
        tc::mma_bf16(tmem, sw128_desc(a + 32 * kk), sw128_mn_desc(b + 2048 * kk, 64 * 128),
                     idesc, i > 0 || kk > 0);
      tc::commit(&empty[st]);
      if (i + kTgStages < nt) {  // refill this stage once its MMAs are done
        if (!mbar_wait_sleep_bounded(&empty[st], (uint32_t)((i / kTgStages) & 1), err)) {
          lost = 1;
          break;
        }
        load(i + kTgStages);
      }
    }
    tc::commit(done);  // every MMA issued so far
  }
  const bool ok = mbar_wait_block(done, 0u, err, lost == 0);
  tc::fence_after_sync();
  const int row = warp * 32 + lane;
  const int64_t m = (int64_t)blockIdx.x * 128 + row;
  const bool live = ok && m < s.M;
  float* dst = part + ((int64_t)blockIdx.y * s.M + m) * 128;
#pragma unroll 1
  for (int c = 0; c < 128; c += 16) {
    float v[16];
    tc::ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
    if (!live) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q)
      *(float4*)(dst + c + 4 * q) = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  }
  // a copy whose wait gave up: wait for every issued stage once more before leaving
  if (threadIdx.x == 0 && lost)
    for (int i = 0; i < kTgStages; ++i) mbar_wait_sleep_bounded(&full[i], 0u, err, 1u);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, 128);
  }
}

// Data gradient of a tap-GEMM layer in two steps.  dcol[m][tap * 64 + ci] = sum_co
// dP[m][co] W[tap * 64 + ci][co] as a GEMM per (m tile, group of four taps): A = the
// dP tile (128 x 128 channels, two SW128 K halves), B = the group's 256 rows of W
// (the same layout: W rows are K-major in co), N = 256, D in TMEM, FP32 out.  Then
// k_conv_col2im gathers dX[voxel][ci] = the sum over the voxel's taps (fixed order)
// of dcol at the output voxel each reaches.  Both operands K-major SW128.
constexpr int kTgDgradSmem = 1024 + 2 * 128 * 128 + 2 * 256 * 128 + 64;

__global__ void __launch_bounds__(128) k_conv_tg_dgrad(const __grid_constant__ CUtensorMap dmap,
                                                       const __grid_constant__ CUtensorMap wmap,
                                                       ConvShape s, float* __restrict__ dcol,
                                                       int* err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* const smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint8_t* const A = smem;                       // [2 K halves][128 rows][128 B]
  uint8_t* const Bt = smem + 2 * 128 * 128;      // [2 K halves][256 rows][128 B]
  uint64_t* const bar = (uint64_t*)(Bt + 2 * 256 * 128);  // [0] loads, [1] MMAs
  uint32_t* const slot = (uint32_t*)(bar + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * 128, g0 = blockIdx.y * 256;
  const int K = 27 * 64;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(slot, 256);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *slot;
  bool lok = true;
  if (threadIdx.x == 0) {
    mbar_expect_tx(&bar[0], 2 * 128 * 128 + 2 * 256 * 128);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      tma_load_2d(A + h * 128 * 128, &dmap, 64 * h, m0, &bar[0]);
      tma_load_2d(Bt + h * 256 * 128, &wmap, 64 * h, g0, &bar[0]);
    }
    lok = mbar_wait_sleep_bounded(&bar[0], 0u, err);
    if (lok) {
      tc::fence_after_sync();
      constexpr uint32_t idesc = tc::idesc_bf16_f32<128, 256>();  // both K-major
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
          tc::mma_bf16(tmem, sw128_desc(smem_u32(A + h * 128 * 128) + 32 * kk),
                       sw128_desc(smem_u32(Bt + h * 256 * 128) + 32 * kk), idesc,
                       h > 0 || kk > 0);
    }
    tc::commit(&bar[1]);  // also without MMAs, so the phase completes
  }
  const bool ok = mbar_wait_block(&bar[1], 0u, err, lok);
  tc::fence_after_sync();
  const int64_t m = (int64_t)m0 + warp * 32 + lane;
  const bool live = ok && m < s.M;
  const int ncol = min(256, K - g0);
  float* dst = dcol + m * K + g0;
#pragma unroll 1
  for (int c = 0; c < 256; c += 16) {
    float v[16];
    tc::ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
    if (!live || c >= ncol) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q)
      *(float4*)(dst + c + 4 * q) = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  }
  // a load wait that gave up: once more, so no copy lands after the block has left
  if (threadIdx.x == 0 && !lok) mbar_wait_sleep_bounded(&bar[0], 0u, err);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, 256);
  }
}

// dX[b, d, h, w, 4 c .. 4 c + 3] = sum over the taps reaching input (d, h, w) -- per
// axis k = 1 from output d / 2 (d even) or k = 0, 2 from outputs (d + 1) / 2, (d - 1) / 2
// (d odd), within the output extent -- of dcol[output][tap * 64 + ci], in tap order.
__global__ void __launch_bounds__(256) k_conv_col2im(const float* __restrict__ dcol, ConvShape s,
                                                     float* __restrict__ dx,
                                                     bf16* __restrict__ dxb) {
  const int64_t n = (int64_t)s.B * s.D * s.H * s.W * 16;  // (voxel, 4-channel group)
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int c4 = (int)(i & 15);
    int64_t v = i >> 4;
    const int w = (int)(v % s.W);
    v /= s.W;
    const int h = (int)(v % s.H);
    v /= s.H;
    const int d = (int)(v % s.D);
    const int b = (int)(v / s.D);
    const int pc[3] = {d, h, w}, no[3] = {s.Do, s.Ho, s.Wo};
    int ks[3][2], os[3][2], nk[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      nk[a] = 0;
      const int p = pc[a];
      if ((p & 1) == 0) {
        if (p / 2 < no[a]) { ks[a][0] = 1; os[a][0] = p / 2; nk[a] = 1; }
      } else {
        if ((p + 1) / 2 < no[a]) { ks[a][nk[a]] = 0; os[a][nk[a]] = (p + 1) / 2; ++nk[a]; }
        ks[a][nk[a]] = 2; os[a][nk[a]] = (p - 1) / 2; ++nk[a];
      }
    }
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i0 = 0; i0 < nk[0]; ++i0)
      for (int i1 = 0; i1 < nk[1]; ++i1)
        for (int i2 = 0; i2 < nk[2]; ++i2) {
          const int tap = (ks[0][i0] * 3 + ks[1][i1]) * 3 + ks[2][i2];
          const int64_t mo = (((int64_t)b * s.Do + os[0][i0]) * s.Ho + os[1][i1]) * s.Wo + os[2][i2];
          const float4 t = *(const float4*)(dcol + mo * (27 * 64) + tap * 64 + 4 * c4);
          acc.x += t.x; acc.y += t.y; acc.z += t.z; acc.w += t.w;
        }
    const int64_t o = (((((int64_t)b * s.D + d) * s.H + h) * s.W + w) * 64) + 4 * c4;
    if (dxb) {
      *(uint2*)(dxb + o) = make_uint2(pack2(__float2bfloat16(acc.x), __float2bfloat16(acc.y)),
                                      pack2(__float2bfloat16(acc.z), __float2bfloat16(acc.w)));
    } else {
      *(float4*)(dx + o) = acc;
    }
  }
}

// Tile geometry of the persistent tap GEMM: Wt = Wo, Ht, Dt, nbt with Wt Ht Dt nbt = 128.
struct TgGeom {
  int wt, ht, dt, nbt;   // tile extents (voxels, rows, planes, images)
  int nh, nd, nbk;       // tiles along h, d and images
};

// Weight + bias gradient of a tap-GEMM layer: block (group, split) accumulates
// dW[(TPG group + t) * CI + ci][co] = sum_m X_tap[m][ci] dP[m][co], t < TPG = 128 / CI
// taps, over the m tiles [split * per, ..) of the forward's tile geometry: A = the
// TPG taps' forward A tiles (the same TMA boxes of x) read MN-major (M = tap x
// channel, MN groups of CI channels one tile apart, K = voxel), B = the tile's dP
// rows (the tile's voxels are consecutive in m), 64-channel SW128 boxes, MN-major;
// eight K = 16 steps per tile, two stages.  The block past the last tap group takes
// an all-ones A: its row 0 is db.  Partials part[split][k][co] with row Kp = db,
// summed in split order by k_sum_splits.
template <int CI, int CO>
struct TgWgrad {
  static constexpr int kTpg = 128 / CI;                   // taps per group
  static constexpr int kGroups = (27 + kTpg - 1) / kTpg;  // + 1 bias block
  static constexpr int kATile = 128 * CI * 2;
  static constexpr int kBTile = 128 * 128;                // one 64-channel dP box
  static constexpr int kStage = kTpg * kATile + (CO / 64) * kBTile;
  static constexpr int kSmem = 1024 + 2 * kStage + 64;
};

template <int CI, int CO>
__global__ void __launch_bounds__(128) k_conv_tg_wgrad(const __grid_constant__ CUtensorMap xmap,
                                                       const __grid_constant__ CUtensorMap dmap,
                                                       ConvShape s, TgGeom g, int per,
                                                       float* __restrict__ part, int* err) {
  using F = TgWgrad<CI, CO>;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* const smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint64_t* const full = (uint64_t*)(smem + 2 * F::kStage);
  uint64_t* const empty = full + 2;
  uint64_t* const done = empty + 2;
  uint32_t* const slot = (uint32_t*)(done + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = blockIdx.x, bias = grp == F::kGroups;
  const int tap0 = grp * F::kTpg;
  const int ntap = bias ? 0 : (27 - tap0 < F::kTpg ? 27 - tap0 : F::kTpg);
  const int64_t mtiles = (int64_t)g.nbk * g.nd * g.nh;
  const int64_t j0 = (int64_t)blockIdx.y * per;
  const int nt = j0 >= mtiles ? 0 : (int)(mtiles - j0 < per ? mtiles - j0 : per);
  if (bias)  // all-ones A in both stages (a constant tile reads the same swizzled or not)
    for (int i = threadIdx.x; i < 2 * F::kTpg * F::kATile / 4; i += 128) {
      const int st = i / (F::kTpg * F::kATile / 4), o = i % (F::kTpg * F::kATile / 4);
      ((uint32_t*)(smem + st * F::kStage))[o] = 0x3F803F80u;
    }
  if (threadIdx.x == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(done, 1);
    fence_mbar_init();
  }
  fence_proxy_async();  // the ones -> the MMA's async-proxy reads
  if (warp == 0) tc::tmem_alloc(slot, CO < 32 ? 32 : CO);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *slot;
  int lost = 0;
  if (threadIdx.x == 0 && nt > 0) {
    auto load = [&](int i) {
      const int st = i & 1;
      int t = (int)(j0 + i);
      const int oh0 = (t % g.nh) * g.ht;
      t /= g.nh;
      const int od0 = (t % g.nd) * g.dt, b0 = (t / g.nd) * g.nbt;
      const int64_t m0 = (((int64_t)b0 * s.Do + od0) * s.Ho + oh0) * s.Wo;
      uint8_t* const a0 = smem + st * F::kStage;
      mbar_expect_tx(&full[st], (uint32_t)(ntap * F::kATile + (CO / 64) * F::kBTile));
      for (int u = 0; u < ntap; ++u) {
        const int tap = tap0 + u, kd = tap / 9, kh = (tap / 3) % 3, kw = tap % 3;
        tma_load_5d(a0 + u * F::kATile, &xmap, 0, kw - 1, 2 * oh0 - 1 + kh, 2 * od0 - 1 + kd, b0,
                    &full[st]);
      }
      for (int h = 0; h < CO / 64; ++h)
        tma_load_2d(a0 + F::kTpg * F::kATile + h * F::kBTile, &dmap, 64 * h, (int)m0, &full[st]);
    };
    load(0);
    if (nt > 1) load(1);
    constexpr uint32_t idesc = tc::idesc_bf16_f32<128, CO>() | (1u << 15) | (1u << 16);
    for (int i = 0; i < nt; ++i) {
      const int st = i & 1;
      if (!mbar_wait_sleep_bounded(&full[st], (uint32_t)((i >> 1) & 1), err)) {
        lost = 1;
        break;
      }
      tc::fence_after_sync();
      const uint32_t a = smem_u32(smem + st * F::kStage), b = a + F::kTpg * F::kATile;
#pragma unroll
      for (int kk = 0; kk < 8; ++kk)  // 128 voxels: eight K = 16 steps of 16 rows
        tc::mma_bf16(tmem, swmn_desc<2 * CI>(a + 32 * CI * kk, F::kATile),
                     swmn_desc<128>(b + 2048 * kk, F::kBTile), idesc, i > 0 || kk > 0);
      tc::commit(&empty[st]);
      if (i + 2 < nt) {
        if (!mbar_wait_sleep_bounded(&empty[st], (uint32_t)((i >> 1) & 1), err)) {
          lost = 1;
          break;
        }
        load(i + 2);
      }
    }
  }
  if (threadIdx.x == 0) tc::commit(done);
  const bool ok = mbar_wait_block(done, 0u, err, lost == 0);
  tc::fence_after_sync();
  float* const pw = part + (int64_t)blockIdx.y * (s.Kp + 1) * CO;
  const int row = warp * 32 + lane;
  int k = -1;
  if (bias)
    k = row == 0 ? s.Kp : -1;
  else if (row / CI < ntap)
    k = (tap0 + row / CI) * CI + row % CI;
  const bool live = ok && k >= 0;
#pragma unroll 1
  for (int c = 0; c < CO; c += 16) {
    float v[16];
    tc::ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
    if (!live) continue;
    if (nt == 0) {
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = 0.f;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
      *(float4*)(pw + (int64_t)k * CO + c + 4 * q) =
          make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  }
  if (threadIdx.x == 0 && lost)
    for (int i = 0; i < 2; ++i) mbar_wait_sleep_bounded(&full[i], 0u, err, 1u);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, CO < 32 ? 32 : CO);
  }
}

// ---------------------------------------------------------------------------
// Persistent tap-GEMM forward for the middle layers (16 -> 32, 32 -> 64 channels).
// A tap's A tile is one TMA box of 128 output voxels (Wt x Ht x Dt x nbt, traversal
// stride 2) whose rows are CI channels (32 or 64 bytes, written with the swizzle of
// that width: the K-major SW32 / SW64 operand, 8-row groups 8 rows apart); B is the
// tap's CI rows of W read MN-major (CO = 32: 64-byte rows, SW64; CO = 64: SW128).
// Warp 4 issues the boxes and the MMAs through a ring over the block's flat (tile,
// tap) sequence; warps 0-3 take a tile's accumulator (two in TMEM, alternating) for
// the bias + GELU epilogue while the next tile's MMAs run.


template <int CI, int CO>
struct TgpFwd {
  static constexpr int kA = 128 * CI * 2;        // A tile bytes
  static constexpr int kB = CI * CO * 2;         // B tile bytes
  static constexpr int kStage = (kA + kB + 1023) / 1024 * 1024;
  static constexpr int kStages = 6;
  static constexpr int kSmem = 1024 + kStages * kStage + 256;
  static constexpr int kCols = 2 * CO <= 32 ? 32 : (2 * CO <= 64 ? 64 : 128);  // two accumulators
  static_assert(kSmem <= 227 * 1024, "stages above the shared-memory limit");
};


template <int CI, int CO>
__global__ void __launch_bounds__(160) k_conv_tgp_fwd(const __grid_constant__ CUtensorMap xmap,
                                                      const __grid_constant__ CUtensorMap wmap,
                                                      ConvShape s, TgGeom g, FwdEp ep, int* err) {
  using F = TgpFwd<CI, CO>;
  constexpr int S = F::kStages;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* const smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint64_t* const full = (uint64_t*)(smem + S * F::kStage);
  uint64_t* const empty = full + S;
  uint64_t* const tfull = empty + S;   // [2] accumulator complete
  uint64_t* const tempty = tfull + 2;  // [2] accumulator read back (one arrival per warp)
  uint64_t* const done = tempty + 2;
  uint32_t* const slot = (uint32_t*)(done + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntiles = g.nbk * g.nd * g.nh;
  const int nloc = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  auto tile_of = [&](int lt, int& b0, int& od0, int& oh0) {
    int t = (int)blockIdx.x + lt * (int)gridDim.x;
    oh0 = (t % g.nh) * g.ht;
    t /= g.nh;
    od0 = (t % g.nd) * g.dt;
    b0 = (t / g.nd) * g.nbt;
  };

  if (threadIdx.x == 0) {
    for (int i = 0; i < S; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&tfull[i], 1);
      mbar_init(&tempty[i], 4);
    }
    mbar_init(done, 1);
    fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(slot, F::kCols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *slot;

  if (warp == 4) {
    if (lane == 0) {
      const int n = nloc * 27;
      auto load = [&](int i) {
        const int st = i % S, tap = i % 27;
        int b0, od0, oh0;
        tile_of(i / 27, b0, od0, oh0);
        const int kd = tap / 9, kh = (tap / 3) % 3, kw = tap % 3;
        uint8_t* const a = smem + st * F::kStage;
        mbar_expect_tx(&full[st], F::kA + F::kB);
        tma_load_5d(a, &xmap, 0, kw - 1, 2 * oh0 - 1 + kh, 2 * od0 - 1 + kd, b0, &full[st]);
        tma_load_2d(a + F::kA, &wmap, 0, tap * CI, &full[st]);
      };
      int issued = 0;  // loads issued (items 0 .. issued - 1)
      for (; issued < n && issued < S; ++issued) load(issued);
      constexpr uint32_t idesc = tc::idesc_bf16_f32<128, CO>() | (1u << 16);  // B MN-major
      bool good = true;
      for (int i = 0; i < n; ++i) {
        const int st = i % S, lt = i / 27, tap = i % 27, acc = lt & 1;
        if (tap == 0 && lt >= 2 &&
            !mbar_wait_sleep_bounded(&tempty[acc], (uint32_t)(((lt >> 1) - 1) & 1), err)) {
          good = false;
          break;
        }
        if (!mbar_wait_sleep_bounded(&full[st], (uint32_t)((i / S) & 1), err)) {
          good = false;
          break;
        }
        tc::fence_after_sync();
        const uint32_t a = smem_u32(smem + st * F::kStage), b = a + F::kA;
#pragma unroll
        for (int kk = 0; kk < CI / 16; ++kk)
          tc::mma_bf16(tmem + (uint32_t)(acc * CO), swk_desc<2 * CI>(a + 32 * kk),
                       swmn_desc<2 * CO>(b + 32 * CO * kk, F::kB), idesc, tap > 0 || kk > 0);
        tc::commit(&empty[st]);
        if (tap == 26) tc::commit(&tfull[acc]);
        // refill the stage of item i - 1 (its MMAs run ahead of item i's)
        if (i >= 1 && issued < n) {
          const int p = i - 1;
          if (!mbar_wait_sleep_bounded(&empty[p % S], (uint32_t)((p / S) & 1), err)) {
            good = false;
            break;
          }
          load(issued++);
        }
      }
      tc::commit(done);
      mbar_wait_sleep_bounded(done, 0u, err);  // every MMA issued is complete
      if (!good)  // copies whose consumer never came: let them land
        for (int i = 0; i < S; ++i) mbar_wait_sleep_bounded(&full[i], 0u, err, 1u);
    }
  } else {  // warps 0..3: epilogue, TMEM lane quarter = warp
    const int row = warp * 32 + lane;
    const int wl = row % g.wt, hl = (row / g.wt) % g.ht, dl = (row / (g.wt * g.ht)) % g.dt;
    const int bl = row / (g.wt * g.ht * g.dt);
    for (int lt = 0; lt < nloc; ++lt) {
      const int acc = lt & 1;
      int ok = 1;
      if (lane == 0) ok = mbar_wait_sleep_bounded(&tfull[acc], (uint32_t)((lt >> 1) & 1), err);
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      if (lane != 0) mbar_wait_bounded(&tfull[acc], (uint32_t)((lt >> 1) & 1), err);
      tc::fence_after_sync();
      int b0, od0, oh0;
      tile_of(lt, b0, od0, oh0);
      const int b = b0 + bl, od = od0 + dl, oh = oh0 + hl;
      const bool live = b < s.B && od < s.Do && oh < s.Ho && wl < s.Wo;
      const int64_t m = (((int64_t)b * s.Do + od) * s.Ho + oh) * s.Wo + wl;
#pragma unroll
      for (int c = 0; c < CO; c += 16) {
        float v[16];
        tc::ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(acc * CO + c), v);
        if (live) ep.put16(m, c, 0, v);
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

// ---------------------------------------------------------------------------
// Per-parity-class tap-GEMM data gradient (32 -> 64 channels, even input extents, so
// every class has the output extents and the forward's tile geometry).  A class
// tile is 128 input voxels (b, 2 j + p) of class p = (pd, ph, pw); each of the
// class's taps (per axis k = 1 for p = 0, k = 0 and 2 for p = 1) reads dP at the
// outputs j + delta (delta = 1 for k = 0, else 0): one stride-1 TMA box of dP (64
// channels = 128-byte rows, K-major SW128; past the extent it reads zero), times the
// tap's 32 rows of W (K-major SW128: N = ci, K = co).  Warp 4 issues through a
// 4-stage ring over the block's flat (class tile, class tap) sequence; warps 0-3
// write dx from one of two TMEM accumulators.
template <int CI, int CO>
struct TgcDgrad {
  static constexpr int kA = 128 * CO * 2;
  static constexpr int kB = CI * CO * 2;
  static constexpr int kStage = (kA + kB + 1023) / 1024 * 1024;
  static constexpr int kStages = 4;
  static constexpr int kSmem = 1024 + kStages * kStage + 256;
  static constexpr int kCols = 2 * CI < 32 ? 32 : 2 * CI;
  static_assert(CO == 64, "dP rows of 128 bytes");
};

// Taps of class c (bits pd ph pw) in order: tap i of 2^(odd axes).
__device__ __forceinline__ void tgc_tap(int c, int i, int& kd, int& kh, int& kw) {
  int k[3];
#pragma unroll
  for (int a = 2; a >= 0; --a) {
    if ((c >> (2 - a)) & 1) {  // odd axis: k = 0 or 2 by the next bit of i
      k[a] = (i & 1) ? 2 : 0;
      i >>= 1;
    } else {
      k[a] = 1;
    }
  }
  kd = k[0];
  kh = k[1];
  kw = k[2];
}

template <int CI, int CO>
__global__ void __launch_bounds__(160) k_conv_tgc_dgrad(const __grid_constant__ CUtensorMap dmap,
                                                        const __grid_constant__ CUtensorMap wmap,
                                                        ConvShape s, TgGeom g,
                                                        float* __restrict__ dx,
                                                        bf16* __restrict__ dxb, int* err) {
  using F = TgcDgrad<CI, CO>;
  constexpr int S = F::kStages;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* const smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint64_t* const full = (uint64_t*)(smem + S * F::kStage);
  uint64_t* const empty = full + S;
  uint64_t* const tfull = empty + S;
  uint64_t* const tempty = tfull + 2;
  uint64_t* const done = tempty + 2;
  uint32_t* const slot = (uint32_t*)(done + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntc = g.nbk * g.nd * g.nh;  // tiles per class
  const int ntiles = 8 * ntc;
  const int nloc = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  // class tile lt of this block: class c and the tile origin (b0, jd0, jh0)
  auto tile_of = [&](int lt, int& c, int& b0, int& jd0, int& jh0) {
    int t = (int)blockIdx.x + lt * (int)gridDim.x;
    c = t / ntc;
    t -= c * ntc;
    jh0 = (t % g.nh) * g.ht;
    t /= g.nh;
    jd0 = (t % g.nd) * g.dt;
    b0 = (t / g.nd) * g.nbt;
  };

  if (threadIdx.x == 0) {
    for (int i = 0; i < S; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&tfull[i], 1);
      mbar_init(&tempty[i], 4);
    }
    mbar_init(done, 1);
    fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(slot, F::kCols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *slot;

  if (warp == 4) {
    if (lane == 0) {
      // flat items: (class tile lt, tap i < 2^popc(c)); the loader runs S items ahead
      int llt = 0, li = 0, lc = 0, lb0 = 0, ljd0 = 0, ljh0 = 0, ln = 0;  // next item to load
      if (nloc > 0) {
        tile_of(0, lc, lb0, ljd0, ljh0);
        ln = 1 << __popc(lc);
      }
      int issued = 0;
      auto load_next = [&]() {  // the item (llt, li) into stage issued % S
        const int st = issued % S;
        int kd, kh, kw;
        tgc_tap(lc, li, kd, kh, kw);
        const int tap = (kd * 3 + kh) * 3 + kw;
        uint8_t* const a = smem + st * F::kStage;
        mbar_expect_tx(&full[st], F::kA + F::kB);
        tma_load_5d(a, &dmap, 0, kw == 0 ? 1 : 0, ljh0 + (kh == 0 ? 1 : 0),
                    ljd0 + (kd == 0 ? 1 : 0), lb0, &full[st]);
        tma_load_2d(a + F::kA, &wmap, 0, tap * CI, &full[st]);
        ++issued;
        if (++li == ln) {  // next class tile
          li = 0;
          if (++llt < nloc) {
            tile_of(llt, lc, lb0, ljd0, ljh0);
            ln = 1 << __popc(lc);
          }
        }
      };
      auto more = [&]() { return llt < nloc; };
      while (issued < S && more()) load_next();
      constexpr uint32_t idesc = tc::idesc_bf16_f32<128, CI>();  // both K-major
      bool good = true;
      int item = 0;
      for (int lt = 0; lt < nloc && good; ++lt) {
        int c, b0, jd0, jh0;
        tile_of(lt, c, b0, jd0, jh0);
        const int nt = 1 << __popc(c), acc = lt & 1;
        if (lt >= 2 &&
            !mbar_wait_sleep_bounded(&tempty[acc], (uint32_t)(((lt >> 1) - 1) & 1), err)) {
          good = false;
          break;
        }
        for (int i = 0; i < nt; ++i, ++item) {
          const int st = item % S;
          if (!mbar_wait_sleep_bounded(&full[st], (uint32_t)((item / S) & 1), err)) {
            good = false;
            break;
          }
          tc::fence_after_sync();
          const uint32_t a = smem_u32(smem + st * F::kStage), b = a + F::kA;
#pragma unroll
          for (int kk = 0; kk < CO / 16; ++kk)
            tc::mma_bf16(tmem + (uint32_t)(acc * CI), swk_desc<128>(a + 32 * kk),
                         swk_desc<128>(b + 32 * kk), idesc, i > 0 || kk > 0);
          tc::commit(&empty[st]);
          if (item >= 1 && more()) {  // refill the stage of the previous item
            const int p = item - 1;
            if (!mbar_wait_sleep_bounded(&empty[p % S], (uint32_t)((p / S) & 1), err)) {
              good = false;
              break;
            }
            load_next();
          }
        }
        tc::commit(&tfull[acc]);
      }
      tc::commit(done);
      mbar_wait_sleep_bounded(done, 0u, err);
      if (!good)
        for (int i = 0; i < S; ++i) mbar_wait_sleep_bounded(&full[i], 0u, err, 1u);
    }
  } else {  // warps 0..3: epilogue
    const int row = warp * 32 + lane;
    const int wl = row % g.wt, hl = (row / g.wt) % g.ht, dl = (row / (g.wt * g.ht)) % g.dt;
    const int bl = row / (g.wt * g.ht * g.dt);
    for (int lt = 0; lt < nloc; ++lt) {
      const int acc = lt & 1;
      int ok = 1;
      if (lane == 0) ok = mbar_wait_sleep_bounded(&tfull[acc], (uint32_t)((lt >> 1) & 1), err);
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      if (lane != 0) mbar_wait_bounded(&tfull[acc], (uint32_t)((lt >> 1) & 1), err);
      tc::fence_after_sync();
      int c, b0, jd0, jh0;
      tile_of(lt, c, b0, jd0, jh0);
      const int b = b0 + bl, jd = jd0 + dl, jh = jh0 + hl;
      const int d = 2 * jd + (c >> 2), h = 2 * jh + ((c >> 1) & 1), w = 2 * wl + (c & 1);
      const bool live = b < s.B && jd < s.Do && jh < s.Ho && wl < s.Wo;
      const int64_t at = ((((int64_t)b * s.D + d) * s.H + h) * s.W + w) * CI;
#pragma unroll
      for (int cc = 0; cc < CI; cc += 16) {
        float v[16];
        tc::ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(acc * CI + cc), v);
        if (!live) continue;
        if (dxb) {
#pragma unroll
          for (int q8 = 0; q8 < 2; ++q8) {
            uint32_t u[4];
#pragma unroll
            for (int j = 0; j < 4; ++j)
              u[j] = pack2(__float2bfloat16(v[8 * q8 + 2 * j]), __float2bfloat16(v[8 * q8 + 2 * j + 1]));
            *(uint4*)(dxb + at + cc + 8 * q8) = make_uint4(u[0], u[1], u[2], u[3]);
          }
        } else {
#pragma unroll
          for (int q4 = 0; q4 < 4; ++q4)
            *(float4*)(dx + at + cc + 4 * q4) =
                make_float4(v[4 * q4], v[4 * q4 + 1], v[4 * q4 + 2], v[4 * q4 + 3]);
        }
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

}  // namespace dm
