// 3x3x3 stride-2 padding-1 3D convolutions (channels-last, BF16 operands, FP32
// accumulation in tensor memory by tcgen05 MMAs) with a fused bias + GELU epilogue,
// and their adjoints.  They run the learned initialiser's encoder (no counterpart in the
// reference).  All three products are implicit GEMMs over one generic tiled
// kernel with gather loaders:
//   forward  C[m, n]  = sum_k  A[m, k] W[k, n]       (A = im2col of x, on the fly)
//   wgrad    dW[k, n] = sum_m  A[m, k] dP[m, n]      (split over m, fixed-order sum;
//                                                   a row of ones appended to A^T
//                                                   gives db in the same product)
//   dgrad    dX[q, c] = sum_t  dP[q(t)] W[t, c]      (one GEMM per stride parity
//                                                   class of the input voxel)
// with m = (b, od, oh, ow), k = ((kd*3 + kh)*3 + kw)*Ci + ci (rows past 27*Ci are
// zero padding up to a multiple of 32), P = pre-activation, dP = dL/dP.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>

#include "../../include/deltamic_b200.h"
#include "band_internal.h"
#include "meshft_internal.h"
#include "tcgen05.cuh"

namespace dm {

using bf16 = __nv_bfloat16;

// Tile: 128 output rows (the MMA's M, one TMEM lane each) x BN columns, reduction
// staged 32 elements at a time (two K = 16 MMAs) through two shared-memory stages.
constexpr int kBM = 128, kBK = 32, kConvThreads = 128;

struct ConvShape {
  int B, D, H, W, Ci;      // input
  int Do, Ho, Wo, Co;      // output
  int K, Kp;               // 27*Ci and its padding to kBK
  int64_t M;               // B*Do*Ho*Wo
  int ci_sh, co_sh;        // log2 of Ci / Co when a power of two, else -1
};

// x / n and x % n for the channel counts: shifts when n is a power of two (the
// loaders' index decomposition runs per gathered element).
__device__ __forceinline__ int ch_div(int x, int n, int sh) { return sh >= 0 ? x >> sh : x / n; }
__device__ __forceinline__ int64_t ch_div(int64_t x, int n, int sh) {
  return sh >= 0 ? x >> sh : x / n;
}

// GELU(x) = x Phi(x) and GELU'(x) = Phi(x) + x phi(x) with the normal CDF from
// erfc by Abramowitz & Stegun 7.1.26: erfc(z) = t (a1 + t (a2 + .. + t a5)) e^{-z^2},
// t = 1 / (1 + p z), z = |x| / sqrt(2) >= 0, |error| <= 1.5e-7 (GELU within 2.2e-7,
// GELU' within 7e-8 of the exact erf forms over the float range; the BF16
// activations resolve 3.9e-3).  e^{-z^2} = e^{-x^2/2} also gives phi.  Phi(x) is
// 1 - erfc(z) / 2 for x >= 0 and erfc(z) / 2 below, so the negative tail keeps its
// relative accuracy.
__device__ __forceinline__ void gelu_parts(float x, float& q, float& e) {
  const float z = fabsf(x) * 0.70710678118654752f;
  const float t = __fdividef(1.f, fmaf(0.3275911f, z, 1.f));
  const float poly =
      t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, 1.061405429f, -1.453152027f), 1.421413741f),
                       -0.284496736f),
               0.254829592f);
  e = __expf(-z * z);
  q = poly * e;  // erfc(z)
}
__device__ __forceinline__ float gelu(float x) {
  float q, e;
  gelu_parts(x, q, e);
  return 0.5f * x * (x >= 0.f ? 2.f - q : q);
}
__device__ __forceinline__ float gelu_grad(float x) {
  float q, e;
  gelu_parts(x, q, e);
  return (x >= 0.f ? 1.f - 0.5f * q : 0.5f * q) + x * e * 0.39894228040143268f;
}

// Output voxel m -> (b, od, oh, ow); 32-bit arithmetic (conv_shape keeps every
// tensor below 2^31 elements).
__device__ __forceinline__ void out_voxel(const ConvShape& s, int64_t m, int& b, int& od, int& oh,
                                          int& ow) {
  uint32_t t = (uint32_t)m;
  ow = (int)(t % (uint32_t)s.Wo); t /= (uint32_t)s.Wo;
  oh = (int)(t % (uint32_t)s.Ho); t /= (uint32_t)s.Ho;
  od = (int)(t % (uint32_t)s.Do);
  b = (int)(t / (uint32_t)s.Do);
}

// Offset of x[b, d, h, w, 0] for the tap (kd, kh, kw) of output voxel m, or -1 in
// the zero padding.
__device__ __forceinline__ int64_t tap_offset(const ConvShape& s, int64_t m, int tap) {
  const int kw = tap % 3, kh = (tap / 3) % 3, kd = tap / 9;
  int b, od, oh, ow;
  out_voxel(s, m, b, od, oh, ow);
  const int d = 2 * od - 1 + kd, h = 2 * oh - 1 + kh, w = 2 * ow - 1 + kw;
  if (d < 0 || d >= s.D || h < 0 || h >= s.H || w < 0 || w >= s.W) return -1;
  return ((((int64_t)b * s.D + d) * s.H + h) * s.W + w) * s.Ci;
}

// im2col element A[m, k] of x (zero outside the volume and in the K padding).
__device__ __forceinline__ bf16 im2col(const bf16* __restrict__ x, const ConvShape& s, int64_t m,
                                       int k) {
  if (k >= s.K) return __float2bfloat16(0.f);
  const int64_t tap = ch_div(k, s.Ci, s.ci_sh);
  const int64_t o = tap_offset(s, m, tap);
  return o < 0 ? __float2bfloat16(0.f) : x[o + k - tap * s.Ci];
}

__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// Eight consecutive reduction elements red0..red0+7 of row ``row`` of A (zero past
// ``rows`` and ``r_end``): one 16-byte load where the loader offers it, else
// element by element.
template <class LA>
__device__ __forceinline__ uint4 gather8_a(const LA& la, int64_t row, int64_t rows, int64_t red0,
                                           int64_t r_end, const int4& info) {
  uint4 v = make_uint4(0u, 0u, 0u, 0u);
  if (row >= rows || red0 >= r_end) return v;
  if (red0 + 8 <= r_end && la.load8(row, red0, info, v)) return v;
  const bf16 z = __float2bfloat16(0.f);
  bf16 e[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) e[j] = red0 + j < r_end ? la(row, red0 + j) : z;
  return make_uint4(pack2(e[0], e[1]), pack2(e[2], e[3]), pack2(e[4], e[5]), pack2(e[6], e[7]));
}

// B[red0..red0+7, col] (zero past r_end).
template <class LB>
__device__ __forceinline__ uint4 gather8_b(const LB& lb, int col, int64_t red0, int64_t r_end) {
  uint4 v = make_uint4(0u, 0u, 0u, 0u);
  if (red0 >= r_end) return v;
  if (red0 + 8 <= r_end && lb.load8(red0, col, v)) return v;
  const bf16 z = __float2bfloat16(0.f);
  bf16 e[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) e[j] = red0 + j < r_end ? lb(red0 + j, col) : z;
  return make_uint4(pack2(e[0], e[1]), pack2(e[2], e[3]), pack2(e[4], e[5]), pack2(e[6], e[7]));
}

// Transposed stage fill: unit (g, mc) supplies rows 8g..8g+7 of reduction column
// mc as one uint4 (element e = row 8g + e), for operands whose contiguous global
// direction runs along the rows.  Each thread stores its eight rows in an order
// rotated by its lane group (lane >> 3 == mc >> 3), so the four lane groups of a
// warp write four different rows of their core matrices: distinct banks.
__device__ __forceinline__ void store_rotated8(bf16* S, int g, int mc, const uint4& v) {
  const int c = mc >> 3;
  const uint32_t w0 = v.x, w1 = v.y, w2 = v.z, w3 = v.w;
  // rw[q] = w[(q + c) & 3]: element j of rw is element (j + 2c) & 7 of v
  const uint32_t rw[4] = {c == 0 ? w0 : c == 1 ? w1 : c == 2 ? w2 : w3,
                          c == 0 ? w1 : c == 1 ? w2 : c == 2 ? w3 : w0,
                          c == 0 ? w2 : c == 1 ? w3 : c == 2 ? w0 : w1,
                          c == 0 ? w3 : c == 1 ? w0 : c == 2 ? w1 : w2};
  bf16* col = S + tc::kmaj32_off(g * 8, mc);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const uint32_t word = rw[j >> 1];
    col[((j + 2 * c) & 7) * 8] = __ushort_as_bfloat16((unsigned short)((j & 1) ? word >> 16 : word));
  }
}

// Up to kMaxGroups / 4 units per thread, all loaded before any is stored.
template <int kMaxGroups, class F>
__device__ __forceinline__ void fill_transposed(bf16* S, int ngroups, F unit) {
  constexpr int kPer = kMaxGroups * 32 / kConvThreads;
  uint4 v[kPer];
  bool use[kPer];
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const int u = threadIdx.x + i * kConvThreads;
    use[i] = u < ngroups * 32 && unit(u >> 5, u & 31, v[i]);
  }
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const int u = threadIdx.x + i * kConvThreads;
    if (use[i]) store_rotated8(S, u >> 5, u & 31, v[i]);
  }
}

// Shared memory of one tile: two stages of A [128 x 32] and B [BN x 32] in the
// K-major no-swizzle layout, two mbarriers, the TMEM address slot and one int4 of
// per-row information (the A loader's, computed once per tile).  The size is
// padded so that the CTAs one SM can hold never ask for more than its 512 TMEM
// columns together (228 KB of shared memory per SM; 16 CTAs of 128 threads at most).
template <int BN>
struct UmmaTile {
  static constexpr int kCols = tc::tmem_cols<BN>();
  static constexpr int kStageA = kBM * kBK;  // elements
  static constexpr int kStageB = BN * kBK;
  static constexpr int kStageBytes = (kStageA + kStageB) * 2;
  static constexpr int kMaxCtas = 512 / kCols;
  static constexpr int kMinSmem = kMaxCtas >= 16 ? 0 : 233472 / (kMaxCtas + 1) + 128;
  static constexpr int kUsed = 2 * kStageBytes + 64 + kBM * 16;  // + per-row info (int4)
  static constexpr int kSmem = ((kUsed > kMinSmem ? kUsed : kMinSmem) + 127) / 128 * 128;
  static_assert(kSmem <= 48 * 1024, "tile shared memory above the default 48 KB");
  static_assert(kStageBytes % 16 == 0, "stage alignment");
};

// Stage of A: the loader's own fill where it has one, else 8-element chunks along
// the reduction.  Chunk e: row (e & 7) + 8 (e >> 5), reduction chunk (e >> 3) & 3 --
// eight lanes store one 128-byte core-matrix column (no bank conflicts), and tiles
// with at most 32 live rows still spread over every thread.  Rows past ``rows``
// are stored as zeros (they only feed accumulator rows that are never read).  All
// of a thread's chunks are loaded before any is stored, so their global loads are
// in flight together.
template <class LA>
__device__ __forceinline__ void fill_a(const LA& la, bf16* As, int64_t row0, int64_t rows,
                                       int64_t k0, int64_t r_end, const int4* rinfo) {
  if (la.fill(As, row0, rows, k0, r_end, rinfo)) return;
  constexpr int kPer = kBM * (kBK / 8) / kConvThreads;
  uint4 v[kPer];
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const int e = threadIdx.x + i * kConvThreads;
    const int r = (e & 7) + ((e >> 5) << 3), kc = (e >> 3) & 3;
    v[i] = row0 + r < rows ? gather8_a(la, row0 + r, rows, k0 + kc * 8, r_end, rinfo[r])
                           : make_uint4(0u, 0u, 0u, 0u);
  }
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const int e = threadIdx.x + i * kConvThreads;
    const int r = (e & 7) + ((e >> 5) << 3), kc = (e >> 3) & 3;
    *(uint4*)(As + tc::kmaj32_off(r, kc * 8)) = v[i];
  }
}

// Stage of B [BN x 32]: the loader's own fill, else chunks along the reduction.
template <int BN, class LB>
__device__ __forceinline__ void fill_b(const LB& lb, bf16* Bs, int64_t k0, int64_t r_end) {
  if (lb.fill(Bs, BN, k0, r_end)) return;
  constexpr int kChunks = BN * (kBK / 8), kPer = (kChunks + kConvThreads - 1) / kConvThreads;
  uint4 v[kPer];
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const int e = threadIdx.x + i * kConvThreads;
    if (e < kChunks) v[i] = gather8_b(lb, e % BN, k0 + (e / BN) * 8, r_end);
  }
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const int e = threadIdx.x + i * kConvThreads;
    if (e < kChunks) *(uint4*)(Bs + tc::kmaj32_off(e % BN, (e / BN) * 8)) = v[i];
  }
}

// Generic tile: C[rows x BN] over a reduction [r_begin, r_end) split by blockIdx.y,
// C = sum_k A[row, k] B[k, col] with A = la(row, k), B = lb(k, col), then
// ep.put16(row, col, split, C[row, col..col+15]).  Every thread gathers its share
// of a stage into shared memory; one thread issues the stage's two tcgen05 MMAs
// into the TMEM accumulator and commits them to the stage's mbarrier, so the next
// stage's gather overlaps them.  Each warp reads its 32 accumulator rows back from
// TMEM for the epilogue.
template <int BN, class LA, class LB, class EP>
__global__ void __launch_bounds__(kConvThreads) k_conv_umma(LA la0, LB lb0, EP ep0, int64_t rows0,
                                                            int64_t red_total0, int64_t red_split,
                                                            int* err) {
  using T = UmmaTile<BN>;
  // blockIdx.z selects a column tile or a sub-problem (the loaders specialise)
  const LA la = la0.at(blockIdx.z);
  const LB lb = lb0.at(blockIdx.z, BN);
  const EP ep = ep0.at(blockIdx.z, BN);
  const int64_t rows = la.rows_at(rows0), red_total = la.red_at(red_total0);
  const int64_t row0 = (int64_t)blockIdx.x * kBM;
  if (row0 >= rows) return;  // whole block, before any TMEM or barrier is set up
  extern __shared__ __align__(128) uint8_t smem[];
  bf16* const As0 = (bf16*)smem;
  bf16* const Bs0 = (bf16*)(smem + T::kStageA * 2);
  uint64_t* const bar = (uint64_t*)(smem + 2 * T::kStageBytes);
  uint32_t* const slot = (uint32_t*)(bar + 2);
  int4* const rinfo = (int4*)(bar + 4);  // 16-byte aligned: bar is
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t r_begin = (int64_t)blockIdx.y * red_split;
  const int64_t r_end = min(red_total, r_begin + red_split);
  const int nk = r_end > r_begin ? (int)((r_end - r_begin + kBK - 1) / kBK) : 0;

  rinfo[threadIdx.x] = la.row_info(row0 + threadIdx.x, rows);
  if (warp == 0) tc::tmem_alloc(slot, T::kCols);
  if (threadIdx.x == 32) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *slot;
  constexpr uint32_t idesc = tc::idesc_bf16_f32<kBM, BN>();

  bool ok = true;
  int issued = 0;
  for (int t = 0; t < nk; ++t) {
    const int s = t & 1;
    bf16* const As = As0 + s * (T::kStageBytes / 2);
    bf16* const Bs = Bs0 + s * (T::kStageBytes / 2);
    // the MMAs of stage t - 2 read this buffer: wait for their commit
    if (t >= 2) ok = mbar_wait_bounded(&bar[s], (uint32_t)(((t - 2) >> 1) & 1), err);
    const int64_t k0 = r_begin + (int64_t)t * kBK;
    fill_a(la, As, row0, rows, k0, r_end, rinfo);
    fill_b<BN>(lb, Bs, k0, r_end);
    fence_proxy_async();  // generic-proxy stores -> the MMA's async-proxy reads
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    if (threadIdx.x == 0) {
      tc::fence_after_sync();
      const uint32_t a0 = smem_u32(As), b0 = smem_u32(Bs);
#pragma unroll
      for (int kk = 0; kk < kBK / 16; ++kk)
        tc::mma_bf16(tmem, tc::smem_desc(a0 + kk * 256), tc::smem_desc(b0 + kk * 256), idesc,
                     t > 0 || kk > 0);
      tc::commit(&bar[s]);
    }
    issued = t + 1;
  }
  // the last commit of each stage not yet waited for: every MMA of the tile is
  // done, and no commit arrives on a barrier after the block has left
  for (int t = issued >= 2 ? issued - 2 : 0; t < issued; ++t)
    ok = mbar_wait_bounded(&bar[t & 1], (uint32_t)((t >> 1) & 1), err) && ok;
  tc::fence_after_sync();
  const int64_t row = row0 + warp * 32 + lane;
#pragma unroll
  for (int c = 0; c < BN; c += 16) {
    float v[16];
    tc::ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
    if (issued == 0) {
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = 0.f;
    }
    if (row < rows) ep.put16(row, c, (int)blockIdx.y, v);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, T::kCols);
  }
}

// ---------------------------------------------------------------------------
// forward

// Loader / epilogue protocol: at(z[, BN]) specialises for blockIdx.z; A loaders
// also give the rows and reduction length of that sub-problem (rows_at, red_at).
struct FwdA {
  const bf16* x;
  ConvShape s;
  bool vec;  // Ci % 8 == 0 and x 16-byte aligned: eight channels of one tap per load
  __device__ FwdA at(int) const { return *this; }
  __device__ int64_t rows_at(int64_t r) const { return r; }
  __device__ int64_t red_at(int64_t r) const { return r; }
  __device__ bf16 operator()(int64_t m, int64_t k) const { return im2col(x, s, m, (int)k); }
  __device__ bool fill(bf16*, int64_t, int64_t, int64_t, int64_t, const int4*) const {
    return false;
  }
  // Row info of output voxel m: the input voxel index of its tap (0, 0, 0) and that
  // tap's coordinates (d0, h0, w0) (possibly -1: the zero padding).
  __device__ int4 row_info(int64_t m, int64_t rows) const {
    if (m >= rows) return make_int4(0, 0, 0, 0);
    int b, od, oh, ow;
    out_voxel(s, m, b, od, oh, ow);
    const int d0 = 2 * od - 1, h0 = 2 * oh - 1, w0 = 2 * ow - 1;
    return make_int4(((b * s.D + d0) * s.H + h0) * s.W + w0, d0, h0, w0);
  }
  __device__ bool load8(int64_t, int64_t k64, const int4& ri, uint4& v) const {
    v = make_uint4(0u, 0u, 0u, 0u);
    const int k = (int)k64;
    if (k >= s.K) return true;
    if (vec) {  // one tap, eight channels
      const int tap = ch_div(k, s.Ci, s.ci_sh), ci = k - tap * s.Ci;
      const int kw = tap % 3, kh = (tap / 3) % 3, kd = tap / 9;
      const int d = ri.y + kd, h = ri.z + kh, w = ri.w + kw;
      if (d >= 0 && d < s.D && h >= 0 && h < s.H && w >= 0 && w < s.W)
        v = *(const uint4*)(x + ((int64_t)ri.x + (kd * s.H + kh) * s.W + kw) * s.Ci + ci);
      return true;
    }
    // Ci < 8: the chunk runs across taps; (ci, kw, kh, kd) decomposed once, then stepped
    const int tap = ch_div(k, s.Ci, s.ci_sh);
    int ci = k - tap * s.Ci, kw = tap % 3, kh = (tap / 3) % 3, kd = tap / 9;
    const bf16 z = __float2bfloat16(0.f);
    bf16 e[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int d = ri.y + kd, h = ri.z + kh, w = ri.w + kw;
      e[j] = (k + j < s.K && d >= 0 && d < s.D && h >= 0 && h < s.H && w >= 0 && w < s.W)
                 ? x[((int64_t)ri.x + (kd * s.H + kh) * s.W + kw) * s.Ci + ci]
                 : z;
      if (++ci == s.Ci) {
        ci = 0;
        if (++kw == 3) {
          kw = 0;
          if (++kh == 3) {
            kh = 0;
            ++kd;
          }
        }
      }
    }
    v = make_uint4(pack2(e[0], e[1]), pack2(e[2], e[3]), pack2(e[4], e[5]), pack2(e[6], e[7]));
    return true;
  }
};
struct WeightB {  // W[k, col0 + n], row-major [Kp, Co]; blockIdx.z = column tile
  const bf16* w;
  int Co;
  int col0;
  __device__ WeightB at(int z, int bn) const { return WeightB{w, Co, z * bn}; }
  __device__ bf16 operator()(int64_t k, int n) const { return w[k * Co + col0 + n]; }
  __device__ bool load8(int64_t, int, uint4&) const { return false; }
  __device__ bool fill(bf16*, int, int64_t, int64_t) const { return false; }
};
struct FwdEp {
  const float* bias;
  float* pre;
  bf16* act;
  int Co;
  int col0;
  bool vec;  // pre and act 16-byte aligned
  __device__ FwdEp at(int z, int bn) const {
    FwdEp e = *this;
    e.col0 = z * bn;
    return e;
  }
  __device__ void put16(int64_t m, int c, int, const float (&v)[16]) const {
    const int n0 = col0 + c;
    float p[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) p[j] = v[j] + (bias ? bias[n0 + j] : 0.f);
    float* pr = pre + m * Co + n0;
    bf16* ar = act + m * Co + n0;
    if (vec) {
#pragma unroll
      for (int q = 0; q < 4; ++q)
        *(float4*)(pr + 4 * q) = make_float4(p[4 * q], p[4 * q + 1], p[4 * q + 2], p[4 * q + 3]);
      uint32_t a[8];
#pragma unroll
      for (int q = 0; q < 8; ++q)
        a[q] = pack2(__float2bfloat16(gelu(p[2 * q])), __float2bfloat16(gelu(p[2 * q + 1])));
      *(uint4*)ar = make_uint4(a[0], a[1], a[2], a[3]);
      *(uint4*)(ar + 8) = make_uint4(a[4], a[5], a[6], a[7]);
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        pr[j] = p[j];
        ar[j] = __float2bfloat16(gelu(p[j]));
      }
    }
  }
};

// Forward with the reduction split over blockIdx.y (few row tiles): each split
// writes its FP32 partial product part[split][m][n]; k_fwd_reduce adds them in
// split order and applies the bias and GELU.
struct FwdSplitEp {
  float* part;
  int64_t stride;  // M * Co
  int Co;
  int col0;
  __device__ FwdSplitEp at(int z, int bn) const {
    FwdSplitEp e = *this;
    e.col0 = z * bn;
    return e;
  }
  __device__ void put16(int64_t m, int c, int split, const float (&v)[16]) const {
    float* r = part + split * stride + m * Co + col0 + c;
#pragma unroll
    for (int q = 0; q < 4; ++q)
      *(float4*)(r + 4 * q) = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  }
};

__global__ void __launch_bounds__(256) k_fwd_reduce(const float* __restrict__ part, int splits,
                                                    int64_t n, int Co,
                                                    const float* __restrict__ bias,
                                                    float* __restrict__ pre,
                                                    bf16* __restrict__ act) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n / 4;
       i += (int64_t)gridDim.x * blockDim.x) {
    float4 v = reinterpret_cast<const float4*>(part)[i];
    for (int k = 1; k < splits; ++k) {
      const float4 q = reinterpret_cast<const float4*>(part + (int64_t)k * n)[i];
      v.x += q.x;
      v.y += q.y;
      v.z += q.z;
      v.w += q.w;
    }
    const int c = (int)((4 * i) % Co);
    if (bias) {
      v.x += bias[c];
      v.y += bias[c + 1];
      v.z += bias[c + 2];
      v.w += bias[c + 3];
    }
    reinterpret_cast<float4*>(pre)[i] = v;
    reinterpret_cast<uint2*>(act)[i] =
        make_uint2(pack2(__float2bfloat16(gelu(v.x)), __float2bfloat16(gelu(v.y))),
                   pack2(__float2bfloat16(gelu(v.z)), __float2bfloat16(gelu(v.w))));
  }
}

// ---------------------------------------------------------------------------
// backward pieces

// dP = dact * GELU'(pre) in BF16; four elements per thread (n is a multiple of 16,
// pointers 16-byte aligned), else one.
__device__ __forceinline__ float ld_grad(const float* g, int64_t i) { return g[i]; }
__device__ __forceinline__ float ld_grad(const bf16* g, int64_t i) {
  return __bfloat162float(g[i]);
}
__device__ __forceinline__ float4 ld_grad4(const float* g, int64_t i) {
  return reinterpret_cast<const float4*>(g)[i];
}
__device__ __forceinline__ float4 ld_grad4(const bf16* g, int64_t i) {
  const uint2 u = reinterpret_cast<const uint2*>(g)[i];
  return make_float4(__uint_as_float(u.x << 16), __uint_as_float(u.x & 0xffff0000u),
                     __uint_as_float(u.y << 16), __uint_as_float(u.y & 0xffff0000u));
}

// dL/dpre = dL/dact * GELU'(pre) in BF16; dL/dact in FP32 or BF16 (TG).
template <bool kVec, class TG>
__global__ void k_gelu_back(const float* __restrict__ pre, const TG* __restrict__ dact,
                            bf16* __restrict__ dpre, int64_t n) {
  if (kVec) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n / 4;
         i += (int64_t)gridDim.x * blockDim.x) {
      const float4 p = ((const float4*)pre)[i], g = ld_grad4(dact, i);
      ((uint2*)dpre)[i] = make_uint2(pack2(__float2bfloat16(g.x * gelu_grad(p.x)),
                                           __float2bfloat16(g.y * gelu_grad(p.y))),
                                     pack2(__float2bfloat16(g.z * gelu_grad(p.z)),
                                           __float2bfloat16(g.w * gelu_grad(p.w))));
    }
  } else {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
      dpre[i] = __float2bfloat16(ld_grad(dact, i) * gelu_grad(pre[i]));
  }
}

struct WgradA {  // A^T[k, m]; row Kp is all ones, so its product row is db
  const bf16* x;
  ConvShape s;
  bool vec;  // Ci % 8 == 0 and x 16-byte aligned: transposed 16-byte gathers
  __device__ WgradA at(int) const { return *this; }
  __device__ int64_t rows_at(int64_t r) const { return r; }
  __device__ int64_t red_at(int64_t r) const { return r; }
  __device__ bf16 operator()(int64_t k, int64_t m) const {
    return k == s.Kp ? __float2bfloat16(1.f) : im2col(x, s, m, (int)k);
  }
  // Row info of row k < K: (ci, kd, kh, kw).
  __device__ int4 row_info(int64_t k64, int64_t) const {
    const int k = (int)k64;
    if (k >= s.K) return make_int4(0, 0, 0, 0);
    const int tap = ch_div(k, s.Ci, s.ci_sh);
    return make_int4(k - tap * s.Ci, tap / 9, (tap / 3) % 3, tap % 3);
  }
  // eight consecutive output voxels m.. at one (tap, ci): decomposed once, then stepped
  __device__ bool load8(int64_t k, int64_t m, const int4& ri, uint4& v) const {
    if (k == s.Kp) {
      v = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);  // BF16 ones
      return true;
    }
    v = make_uint4(0u, 0u, 0u, 0u);
    if (k >= s.K) return true;
    int b, od, oh, ow;
    out_voxel(s, m, b, od, oh, ow);
    const bf16 z = __float2bfloat16(0.f);
    bf16 e[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int d = 2 * od - 1 + ri.y, h = 2 * oh - 1 + ri.z, w = 2 * ow - 1 + ri.w;
      e[j] = (b < s.B && d >= 0 && d < s.D && h >= 0 && h < s.H && w >= 0 && w < s.W)
                 ? x[((((int64_t)b * s.D + d) * s.H + h) * s.W + w) * s.Ci + ri.x]
                 : z;
      if (++ow == s.Wo) {
        ow = 0;
        if (++oh == s.Ho) {
          oh = 0;
          if (++od == s.Do) {
            od = 0;
            ++b;
          }
        }
      }
    }
    v = make_uint4(pack2(e[0], e[1]), pack2(e[2], e[3]), pack2(e[4], e[5]), pack2(e[6], e[7]));
    return true;
  }
  // Ci % 8 == 0: lane = reduction column (its voxel decomposed once per stage); per
  // row group of eight k (one tap, eight channels) one 16-byte load, stored transposed
  __device__ bool fill(bf16* As, int64_t row0, int64_t rows, int64_t m0, int64_t r_end,
                       const int4* rinfo) const {
    if (!vec) return false;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t m = m0 + lane;
    const bool mv = m < r_end;
    int b = 0, od = 0, oh = 0, ow = 0;
    if (mv) out_voxel(s, m, b, od, oh, ow);
    const int d0 = 2 * od - 1, h0 = 2 * oh - 1, w0 = 2 * ow - 1;
    const int vbase = ((b * s.D + d0) * s.H + h0) * s.W + w0;
    constexpr int kPer = kBM / 8 / (kConvThreads / 32);
    uint4 v[kPer];
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int g = warp + (kConvThreads / 32) * i;
      const int64_t k = row0 + g * 8;
      v[i] = make_uint4(0u, 0u, 0u, 0u);
      if (mv && k < rows) {
        if (k == s.Kp) {
          v[i].x = 0x3F80u;  // row Kp: one; rows Kp+1.. are past ``rows``
        } else if (k < s.K) {
          const int4 ri = rinfo[g * 8];
          const int d = d0 + ri.y, h = h0 + ri.z, w = w0 + ri.w;
          if (d >= 0 && d < s.D && h >= 0 && h < s.H && w >= 0 && w < s.W)
            v[i] = *(const uint4*)(x + ((int64_t)vbase + (ri.y * s.H + ri.z) * s.W + ri.w) *
                                           s.Ci + ri.x);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int g = warp + (kConvThreads / 32) * i;
      if (row0 + g * 8 < rows) store_rotated8(As, g, lane, v[i]);
    }
    return true;
  }
};
struct DpreB {  // dP[m, n]
  const bf16* dp;
  int Co;
  bool vec;  // dp 16-byte aligned (Co is a multiple of 8): eight channels per load
  __device__ DpreB at(int, int) const { return *this; }
  __device__ bf16 operator()(int64_t m, int n) const { return dp[m * Co + n]; }
  __device__ bool load8(int64_t, int, uint4&) const { return false; }
  __device__ bool fill(bf16* Bs, int bn, int64_t m0, int64_t r_end) const {
    if (!vec) return false;
    fill_transposed<128 / 8>(Bs, bn / 8, [&](int g, int mc, uint4& v) {
      const int64_t m = m0 + mc;
      v = make_uint4(0u, 0u, 0u, 0u);
      if (m < r_end) v = *(const uint4*)(dp + m * Co + g * 8);
      return true;
    });
    return true;
  }
};
struct WgradEp {  // partial[split][k][n] (16-byte aligned workspace rows)
  float* part;
  int64_t stride;  // (Kp + 1) * Co
  int Co;
  __device__ WgradEp at(int, int) const { return *this; }
  __device__ void put16(int64_t k, int c, int split, const float (&v)[16]) const {
    float* r = part + split * stride + k * Co + c;
#pragma unroll
    for (int q = 0; q < 4; ++q)
      *(float4*)(r + 4 * q) = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  }
};

// Fixed-order sum of the split partials [split][Kp + 1][Co]: rows < Kp into dw,
// row Kp (the ones row) into db.  Block (32, 8): x runs along the outputs
// (coalesced), y takes every eighth split; the eight partial sums are added in
// order of y.
__global__ void __launch_bounds__(256) k_sum_splits(const float* __restrict__ part, int splits,
                                                    int64_t nw, int Co, float* __restrict__ dw,
                                                    float* __restrict__ db) {
  __shared__ float sh[8][33];
  const int64_t n = nw + Co;
  const int64_t i = (int64_t)blockIdx.x * 32 + threadIdx.x;
  float s = 0.f;
  if (i < n)
    for (int k = threadIdx.y; k < splits; k += 8) s += part[k * n + i];
  sh[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && i < n) {
    float t = sh[0][threadIdx.x];
#pragma unroll
    for (int y = 1; y < 8; ++y) t += sh[y][threadIdx.x];
    if (i < nw)
      dw[i] = t;
    else
      db[i - nw] = t;
  }
}

// dgrad for the input voxels of one stride-parity class (pd, ph, pw): per axis an
// even coordinate d takes tap 1 (od = d/2), an odd one taps 0 and 2
// (od = (d+1)/2, (d-1)/2).  The eight classes run in one launch, blockIdx.z = class.
struct Cls {
  int p[3];      // parity per axis
  int n[3];      // class extent per axis
  int nt[3];     // taps per axis (1 or 2)
  int T;         // taps in the class
  int64_t rows;  // B * n0 * n1 * n2 (0: empty class)
  int64_t red;   // T * Co rounded up to kBK
};
struct ClsSet {
  Cls c[8];
};

// Class z of a set held in kernel parameters (constant indices: no local copy).
__device__ __forceinline__ Cls pick_cls(const ClsSet& set, int z) {
  switch (z) {
    case 0: return set.c[0];
    case 1: return set.c[1];
    case 2: return set.c[2];
    case 3: return set.c[3];
    case 4: return set.c[4];
    case 5: return set.c[5];
    case 6: return set.c[6];
    default: return set.c[7];
  }
}

__device__ __forceinline__ void cls_tap(const Cls& c, int t, int kk[3]) {
  // taps per axis are 1 or 2: shifts and masks
  const int s2 = c.nt[2] - 1, s1 = c.nt[1] - 1;
  const int tw = t & s2, th = (t >> s2) & s1, td = t >> (s2 + s1);
  const int tt[3] = {td, th, tw};
#pragma unroll
  for (int a = 0; a < 3; ++a) kk[a] = c.p[a] == 0 ? 1 : (tt[a] == 0 ? 0 : 2);
}

// Input voxel of class row q: (b, d, h, w).
__device__ __forceinline__ void cls_voxel(const Cls& c, int64_t q, int& b, int& d, int& h,
                                          int& w) {
  uint32_t u = (uint32_t)q;
  const int iw = (int)(u % (uint32_t)c.n[2]); u /= (uint32_t)c.n[2];
  const int ih = (int)(u % (uint32_t)c.n[1]); u /= (uint32_t)c.n[1];
  const int id = (int)(u % (uint32_t)c.n[0]);
  b = (int)(u / (uint32_t)c.n[0]);
  d = 2 * id + c.p[0];
  h = 2 * ih + c.p[1];
  w = 2 * iw + c.p[2];
}

struct DgradA {  // A[q, (tap, co)] = dP at the output voxel reached through the tap
  const bf16* dp;
  ConvShape s;
  ClsSet set;  // the eight classes (kernel parameter)
  Cls c;
  bool vec;  // dp 16-byte aligned (Co is a multiple of 8): eight channels per load
  __device__ DgradA at(int z) const {
    DgradA a = *this;
    a.c = pick_cls(set, z);
    return a;
  }
  __device__ int64_t rows_at(int64_t) const { return c.rows; }
  __device__ int64_t red_at(int64_t) const { return c.red; }
  // Offset of dP[voxel reached from input voxel q through tap t, 0], or -1 outside.
  __device__ int64_t offset(int64_t q, int t) const {
    int kk[3], b, d, h, w;
    cls_tap(c, t, kk);
    cls_voxel(c, q, b, d, h, w);
    const int od = (d + 1 - kk[0]) >> 1, oh = (h + 1 - kk[1]) >> 1, ow = (w + 1 - kk[2]) >> 1;
    if (od < 0 || od >= s.Do || oh < 0 || oh >= s.Ho || ow < 0 || ow >= s.Wo) return -1;
    return ((((int64_t)b * s.Do + od) * s.Ho + oh) * s.Wo + ow) * s.Co;
  }
  __device__ bf16 operator()(int64_t q, int64_t r) const {
    const int t = (int)ch_div(r, s.Co, s.co_sh);
    if (t >= c.T) return __float2bfloat16(0.f);
    const int64_t o = offset(q, t);
    return o < 0 ? __float2bfloat16(0.f) : dp[o + r - (int64_t)t * s.Co];
  }
  // Row info of class row q: its input voxel (b, d, h, w).
  __device__ int4 row_info(int64_t q, int64_t rows) const {
    if (q >= rows) return make_int4(0, 0, 0, 0);
    int b, d, h, w;
    cls_voxel(c, q, b, d, h, w);
    return make_int4(b, d, h, w);
  }
  __device__ bool load8(int64_t, int64_t r64, const int4& ri, uint4& v) const {
    if (!vec) return false;
    v = make_uint4(0u, 0u, 0u, 0u);
    const int r = (int)r64, t = ch_div(r, s.Co, s.co_sh);
    if (t >= c.T) return true;
    int kk[3];
    cls_tap(c, t, kk);
    const int od = (ri.y + 1 - kk[0]) >> 1, oh = (ri.z + 1 - kk[1]) >> 1,
              ow = (ri.w + 1 - kk[2]) >> 1;
    if (od < 0 || od >= s.Do || oh < 0 || oh >= s.Ho || ow < 0 || ow >= s.Wo) return true;
    v = *(const uint4*)(dp + ((((int64_t)ri.x * s.Do + od) * s.Ho + oh) * s.Wo + ow) * s.Co +
                        (r - t * s.Co));
    return true;
  }
  __device__ bool fill(bf16*, int64_t, int64_t, int64_t, int64_t, const int4*) const {
    return false;
  }
};
struct DgradB {  // B[(tap, co), ci] = W[(k(tap), ci), co]
  const bf16* w;
  ConvShape s;
  ClsSet set;
  Cls c;
  bool vec;  // w 16-byte aligned (Co is a multiple of 8): eight co per load
  __device__ DgradB at(int z, int) const {
    DgradB b = *this;
    b.c = pick_cls(set, z);
    return b;
  }
  __device__ int64_t offset(int t, int ci) const {
    int kk[3];
    cls_tap(c, t, kk);
    const int tap = (kk[0] * 3 + kk[1]) * 3 + kk[2];
    return ((int64_t)tap * s.Ci + ci) * s.Co;
  }
  __device__ bf16 operator()(int64_t r, int ci) const {
    const int t = (int)ch_div(r, s.Co, s.co_sh);
    if (t >= c.T || ci >= s.Ci) return __float2bfloat16(0.f);
    return w[offset(t, ci) + r - (int64_t)t * s.Co];
  }
  __device__ bool load8(int64_t r, int ci, uint4& v) const {
    if (!vec) return false;
    v = make_uint4(0u, 0u, 0u, 0u);
    const int t = (int)ch_div(r, s.Co, s.co_sh);
    if (t >= c.T || ci >= s.Ci) return true;
    v = *(const uint4*)(w + offset(t, ci) + r - (int64_t)t * s.Co);
    return true;
  }
  __device__ bool fill(bf16*, int, int64_t, int64_t) const { return false; }
};
struct DgradEp {
  float* dx;
  bf16* dxb;  // BF16 output instead of dx when not NULL
  ConvShape s;
  ClsSet set;
  Cls c;
  bool vec;  // dx 16-byte aligned and Ci a multiple of 16
  __device__ DgradEp at(int z, int) const {
    DgradEp e = *this;
    e.c = pick_cls(set, z);
    return e;
  }
  __device__ void put16(int64_t q, int c0, int, const float (&v)[16]) const {
    if (c0 >= s.Ci) return;
    int b, d, h, w;
    cls_voxel(c, q, b, d, h, w);
    const int64_t at = ((((int64_t)b * s.D + d) * s.H + h) * s.W + w) * s.Ci + c0;
    if (dxb) {
      bf16* r = dxb + at;
      if (vec) {
#pragma unroll
        for (int q8 = 0; q8 < 2; ++q8) {
          uint32_t u[4];
#pragma unroll
          for (int j = 0; j < 4; ++j)
            u[j] = pack2(__float2bfloat16(v[8 * q8 + 2 * j]),
                         __float2bfloat16(v[8 * q8 + 2 * j + 1]));
          *(uint4*)(r + 8 * q8) = make_uint4(u[0], u[1], u[2], u[3]);
        }
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j)
          if (c0 + j < s.Ci) r[j] = __float2bfloat16(v[j]);
      }
      return;
    }
    float* r = dx + at;
    if (vec) {
#pragma unroll
      for (int q4 = 0; q4 < 4; ++q4)
        *(float4*)(r + 4 * q4) =
            make_float4(v[4 * q4], v[4 * q4 + 1], v[4 * q4 + 2], v[4 * q4 + 3]);
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j)
        if (c0 + j < s.Ci) r[j] = v[j];
    }
  }
};

}  // namespace dm

#include "conv_fp.cuh"
#include "conv_s2d.cuh"
#include "conv_tg.cuh"

namespace dm {

// ---------------------------------------------------------------------------
// launchers

// Status word of the convolution kernels (bounded waits that gave up), one per
// device; its device address is looked up per device (with that device current).
__device__ int g_conv_status;

constexpr int kConvMaxDevices = 64;
static std::atomic<int*> g_conv_status_addr[kConvMaxDevices];

static int* conv_status_ptr() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kConvMaxDevices) return nullptr;
  int* p = g_conv_status_addr[dev].load();
  if (!p) {
    void* a = nullptr;
    if (cudaGetSymbolAddress(&a, g_conv_status) != cudaSuccess) return nullptr;
    p = (int*)a;
    g_conv_status_addr[dev].store(p);
  }
  return p;
}

// rows: the largest sub-problem's rows (grid x); nz sub-problems or column tiles.
template <int BN, class LA, class LB, class EP>
static void umma_launch(LA la, LB lb, EP ep, int64_t rows, int64_t red, int64_t red_split,
                        int splits, int nz, cudaStream_t st) {
  const dim3 grid((unsigned)((rows + kBM - 1) / kBM), (unsigned)splits, (unsigned)nz);
  k_conv_umma<BN><<<grid, kConvThreads, UmmaTile<BN>::kSmem, st>>>(la, lb, ep, rows, red,
                                                                    red_split, conv_status_ptr());
}

template <class LA, class LB, class EP>
static void gemm_launch(int bn, LA la, LB lb, EP ep, int64_t rows, int64_t red, int64_t red_split,
                        int splits, int nz, cudaStream_t st) {
  switch (bn) {
    case 16: umma_launch<16>(la, lb, ep, rows, red, red_split, splits, nz, st); break;
    case 32: umma_launch<32>(la, lb, ep, rows, red, red_split, splits, nz, st); break;
    case 64: umma_launch<64>(la, lb, ep, rows, red, red_split, splits, nz, st); break;
    default: umma_launch<128>(la, lb, ep, rows, red, red_split, splits, nz, st); break;
  }
  count_launches(1);
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// ---------------------------------------------------------------------------
// Single-channel input (the encoder's first layer, Ci = 1): the reduction is only
// 27 taps long, so an implicit GEMM spends its time gathering 2-byte elements.
// These direct kernels stage each tile's input footprint once in shared memory
// instead -- a tile is (b, od, 8 output rows, 32 output columns); its input is 3
// planes x 17 rows x 65 columns -- and stream the outputs (HBM-bound: 2 B read and
// 6 Co B written per output voxel in the forward).  Products and sums in FP32 on
// the same BF16 inputs.

constexpr int kC1TH = 8, kC1TW = 32;                       // output tile rows x columns
constexpr int kC1IH = 2 * kC1TH + 1, kC1IW = 2 * kC1TW + 1;  // input footprint

struct C1Tile {
  int b, od, oh0, ow0;
};

__device__ __forceinline__ C1Tile c1_tile(const ConvShape& s, int64_t t) {
  const int nw = (s.Wo + kC1TW - 1) / kC1TW, nh = (s.Ho + kC1TH - 1) / kC1TH;
  C1Tile r;
  r.ow0 = (int)(t % nw) * kC1TW;
  t /= nw;
  r.oh0 = (int)(t % nh) * kC1TH;
  t /= nh;
  r.od = (int)(t % s.Do);
  r.b = (int)(t / s.Do);
  return r;
}

__device__ __forceinline__ int64_t c1_tiles(const ConvShape& s) {
  return (int64_t)s.B * s.Do * ((s.Ho + kC1TH - 1) / kC1TH) * ((s.Wo + kC1TW - 1) / kC1TW);
}

// Input footprint of a tile in shared memory, columns de-interleaved: row r of
// plane p holds the even columns 0, 2, .., 64 at [0, 33) and the odd columns
// 1, 3, .., 63 at [34, 66), rows kC1RS apart, planes kC1PS apart (zero outside the
// volume).  Output column tx, tap kw then reads offset kC1Col[kw] + tx: consecutive
// across the lanes of a forward warp (one voxel per lane), and, with the strides
// = 3 and 9 (mod 32) banks, 27 distinct banks across the lanes of a weight-gradient
// warp (one tap per lane).
constexpr int kC1RS = 67, kC1PS = 1161, kC1XS = 3 * kC1PS;

__device__ __forceinline__ int c1_col(int kw) { return kw == 0 ? 0 : (kw == 1 ? 34 : 1); }

__device__ __forceinline__ void c1_load(const bf16* __restrict__ x, const ConvShape& s,
                                        const C1Tile& tl, float* xs) {
  // warp w takes footprint rows w, w + 8, ...; lane l the columns 2l + 1, 2l + 2 (one
  // aligned pair of input columns, w = 2 ow0 + 2l) and lane 0 also column 0
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kRows = 3 * kC1IH;
  for (int row = warp; row < kRows; row += 8) {
    const int pz = row / kC1IH, r = row - pz * kC1IH;
    const int d = 2 * tl.od - 1 + pz, h = 2 * tl.oh0 - 1 + r;
    float* xr = xs + pz * kC1PS + r * kC1RS;
    const bool in_dh = d >= 0 && d < s.D && h >= 0 && h < s.H;
    const bf16* src = x + (((int64_t)tl.b * s.D + (in_dh ? d : 0)) * s.H + (in_dh ? h : 0)) * s.W;
    const int w0 = 2 * tl.ow0 + 2 * lane;  // columns 2l + 1 and 2l + 2 of the footprint
    float odd = 0.f, even = 0.f;
    if (in_dh) {
      // one 4-byte load when the pair is 4-byte aligned (even rows, aligned base)
      if (w0 + 1 < s.W && (s.W & 1) == 0 && ((uintptr_t)x & 3) == 0) {
        const uint32_t u = *reinterpret_cast<const uint32_t*>(src + w0);
        odd = __uint_as_float(u << 16);
        even = __uint_as_float(u & 0xffff0000u);
      } else {
        if (w0 < s.W) odd = __bfloat162float(src[w0]);
        if (w0 + 1 < s.W) even = __bfloat162float(src[w0 + 1]);
      }
    }
    xr[34 + lane] = odd;       // footprint column 2l + 1
    xr[lane + 1] = even;       // footprint column 2l + 2
    if (lane == 0) {           // footprint column 0: input column 2 ow0 - 1
      const int wl = 2 * tl.ow0 - 1;
      xr[0] = (in_dh && wl >= 0) ? __bfloat162float(src[wl]) : 0.f;
    }
  }
}

// pre = x * W + bias, act = GELU(pre) for one output voxel per thread.
template <int CO>
__global__ void __launch_bounds__(256) k_conv1_fwd(const bf16* __restrict__ x, ConvShape s,
                                                   const bf16* __restrict__ w,
                                                   const float* __restrict__ bias,
                                                   float* __restrict__ pre,
                                                   bf16* __restrict__ act) {
  __shared__ float xs[kC1XS];
  __shared__ __align__(16) float ws[27][CO];
  __shared__ __align__(16) float bs[CO];
  for (int i = threadIdx.x; i < 27 * CO; i += blockDim.x)
    ws[i / CO][i % CO] = __bfloat162float(w[i]);  // rows 0..26 of W[Kp][Co]
  if (threadIdx.x < CO) bs[threadIdx.x] = bias ? bias[threadIdx.x] : 0.f;
  const C1Tile tl = c1_tile(s, blockIdx.x);
  c1_load(x, s, tl, xs);
  __syncthreads();
  const int ty = threadIdx.x / kC1TW, tx = threadIdx.x % kC1TW;
  const int oh = tl.oh0 + ty, ow = tl.ow0 + tx;
  if (oh >= s.Ho || ow >= s.Wo) return;
  // channel pairs on the paired FP32 path (two FMAs per instruction)
  float2 acc2[CO / 2];
#pragma unroll
  for (int c = 0; c < CO / 2; ++c) acc2[c] = make_float2(bs[2 * c], bs[2 * c + 1]);
#pragma unroll
  for (int kd = 0; kd < 3; ++kd)
#pragma unroll
    for (int kh = 0; kh < 3; ++kh)
#pragma unroll
      for (int kw = 0; kw < 3; ++kw) {
        const float xv = xs[kd * kC1PS + (2 * ty + kh) * kC1RS + c1_col(kw) + tx];
        const float2 x2 = make_float2(xv, xv);
        const int tap = (kd * 3 + kh) * 3 + kw;
        const float4* w4 = reinterpret_cast<const float4*>(&ws[tap][0]);
#pragma unroll
        for (int q = 0; q < CO / 4; ++q) {
          const float4 wv = w4[q];
          acc2[2 * q] = __ffma2_rn(x2, make_float2(wv.x, wv.y), acc2[2 * q]);
          acc2[2 * q + 1] = __ffma2_rn(x2, make_float2(wv.z, wv.w), acc2[2 * q + 1]);
        }
      }
  float acc[CO];
#pragma unroll
  for (int c = 0; c < CO / 2; ++c) {
    acc[2 * c] = acc2[c].x;
    acc[2 * c + 1] = acc2[c].y;
  }
  const int64_t m = (((int64_t)tl.b * s.Do + tl.od) * s.Ho + oh) * s.Wo + ow;
  float4* pp = reinterpret_cast<float4*>(pre + m * CO);
  uint4* ap = reinterpret_cast<uint4*>(act + m * CO);
#pragma unroll
  for (int q = 0; q < CO / 4; ++q) pp[q] = make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2],
                                                       acc[4 * q + 3]);
#pragma unroll
  for (int q = 0; q < CO / 8; ++q) {
    uint32_t u[4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
      u[j] = pack2(__float2bfloat16(gelu(acc[8 * q + 2 * j])),
                   __float2bfloat16(gelu(acc[8 * q + 2 * j + 1])));
    ap[q] = make_uint4(u[0], u[1], u[2], u[3]);
  }
}

// Weight and bias gradient partials: block g sums its tiles (g, g + G, ...) into
// part[g][(Kp + 1) * CO] (rows 0..26 taps, 27..Kp-1 zero, row Kp the bias);
// k_sum_splits adds the blocks in order.  dP is the BF16 dL/dpre of k_gelu_back.
// Lane l of every warp owns tap l (l = 27: the bias, input 1; lanes 28..31 idle)
// and all CO channels; warp w takes the tile's voxels w, w + 8, ..: per voxel one
// shared-memory read of the input (27 banks) and CO / 4 broadcast 16-byte reads of
// the voxel's dP row.  The eight warps' sums are added in warp order at the end.
template <int CO>
__global__ void __launch_bounds__(256) k_conv1_wgrad(const bf16* __restrict__ x, ConvShape s,
                                                     const bf16* __restrict__ dp,
                                                     float* __restrict__ part) {
  constexpr int NV = kC1TH * kC1TW;
  // dP rows, then the footprint; after the last tile the warps' sums reuse the space
  __shared__ __align__(16) float sm[NV * CO + kC1XS];
  static_assert(8 * 28 * CO <= NV * CO + kC1XS, "reduction area");
  float* ds = sm;
  float* xs = sm + NV * CO;
  float* red = sm;  // [8][28 * CO], after the loop
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tap = min(lane, 27);
  const int kd = tap / 9, kh = (tap / 3) % 3, kw = tap % 3;
  const int xoff = kd * kC1PS + kh * kC1RS + c1_col(kw);
  float2 acc2[CO / 2];  // channel pairs on the paired FP32 path
#pragma unroll
  for (int c = 0; c < CO / 2; ++c) acc2[c] = make_float2(0.f, 0.f);
  const int64_t ntl = c1_tiles(s);
  for (int64_t t = blockIdx.x; t < ntl; t += gridDim.x) {
    const C1Tile tl = c1_tile(s, t);
    __syncthreads();  // the previous tile's reads are done
    c1_load(x, s, tl, xs);
    // dP rows of the tile's voxels, 16-byte loads (8 channels each)
    constexpr int NQ = NV * CO / 8;
#pragma unroll
    for (int u = 0; u < (NQ + 255) / 256; ++u) {
      const int q = threadIdx.x + 256 * u;
      if (q >= NQ) continue;
      const int v = q / (CO / 8), c0 = (q % (CO / 8)) * 8;
      const int oh = tl.oh0 + v / kC1TW, ow = tl.ow0 + v % kC1TW;
      uint4 g = make_uint4(0u, 0u, 0u, 0u);
      if (oh < s.Ho && ow < s.Wo)
        g = *reinterpret_cast<const uint4*>(
            dp + ((((int64_t)tl.b * s.Do + tl.od) * s.Ho + oh) * s.Wo + ow) * CO + c0);
      const uint32_t gw[4] = {g.x, g.y, g.z, g.w};
      float4* d4 = reinterpret_cast<float4*>(ds + v * CO + c0);
      float f[8];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        f[2 * j] = __uint_as_float(gw[j] << 16);
        f[2 * j + 1] = __uint_as_float(gw[j] & 0xffff0000u);
      }
      d4[0] = make_float4(f[0], f[1], f[2], f[3]);
      d4[1] = make_float4(f[4], f[5], f[6], f[7]);
    }
    __syncthreads();
    for (int v = warp; v < NV; v += 8) {
      const int ty = v / kC1TW, tx = v % kC1TW;
      const float xv = lane < 27 ? xs[xoff + 2 * ty * kC1RS + tx] : (lane == 27 ? 1.f : 0.f);
      const float2 x2 = make_float2(xv, xv);
      const float4* d4 = reinterpret_cast<const float4*>(ds + v * CO);
#pragma unroll
      for (int q = 0; q < CO / 4; ++q) {
        const float4 g = d4[q];
        acc2[2 * q] = __ffma2_rn(x2, make_float2(g.x, g.y), acc2[2 * q]);
        acc2[2 * q + 1] = __ffma2_rn(x2, make_float2(g.z, g.w), acc2[2 * q + 1]);
      }
    }
  }
  float acc[CO];
#pragma unroll
  for (int c = 0; c < CO / 2; ++c) {
    acc[2 * c] = acc2[c].x;
    acc[2 * c + 1] = acc2[c].y;
  }
  __syncthreads();  // every warp is done with ds / xs
  if (lane < 28) {
#pragma unroll
    for (int c = 0; c < CO; ++c) red[warp * 28 * CO + lane * CO + c] = acc[c];
  }
  __syncthreads();
  float* out = part + (int64_t)blockIdx.x * (s.Kp + 1) * CO;
  for (int o = threadIdx.x; o < 28 * CO; o += blockDim.x) {
    float a = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) a += red[k * 28 * CO + o];
    if (o < 27 * CO) out[o] = a;
    else out[(int64_t)s.Kp * CO + (o - 27 * CO)] = a;
  }
  for (int o = 27 * CO + threadIdx.x; o < s.Kp * CO; o += blockDim.x) out[o] = 0.f;
}

static bool conv1_direct(const ConvShape& s) { return s.Ci == 1 && (s.Co == 16 || s.Co == 32); }

static int64_t conv1_tiles_host(const ConvShape& s) {
  return (int64_t)s.B * s.Do * ((s.Ho + kC1TH - 1) / kC1TH) * ((s.Wo + kC1TW - 1) / kC1TW);
}

static int pad_cols(int c) { return c <= 16 ? 16 : (c <= 32 ? 32 : (c <= 64 ? 64 : 128)); }

bool conv_shape(int B, int D, int H, int W, int Ci, int Co, ConvShape& s) {
  if (B <= 0 || D <= 0 || H <= 0 || W <= 0 || Ci <= 0 || Co <= 0 || Co > 128 || Ci > 128)
    return false;
  if (Co != 16 && Co != 32 && Co != 64 && Co != 128) return false;
  // every tensor below 2^31 elements (32-bit voxel arithmetic in the kernels)
  if ((int64_t)B * D * H * W * std::max(Ci, Co) >= ((int64_t)1 << 31)) return false;
  s.B = B; s.D = D; s.H = H; s.W = W; s.Ci = Ci; s.Co = Co;
  s.Do = (D + 1) / 2; s.Ho = (H + 1) / 2; s.Wo = (W + 1) / 2;
  s.K = 27 * Ci;
  s.Kp = (s.K + kBK - 1) / kBK * kBK;
  s.M = (int64_t)B * s.Do * s.Ho * s.Wo;
  auto lg = [](int n) { return (n & (n - 1)) == 0 ? __builtin_ctz((unsigned)n) : -1; };
  s.ci_sh = lg(Ci);
  s.co_sh = lg(Co);
  return true;
}

// Blocks per SM the tile kernel reaches: shared memory allows 8-10 up to BN = 64,
// the 512 TMEM columns 4 at BN = 128.
static int tile_blocks_per_sm(int bn) { return bn >= 128 ? 4 : 8; }

static int wgrad_splits(const ConvShape& s) {
  const int64_t row_tiles = (s.Kp + 1 + kBM - 1) / kBM;
  int64_t sp = std::max<int64_t>(1, (int64_t)148 * tile_blocks_per_sm(s.Co) / row_tiles);
  sp = std::min<int64_t>(sp, std::max<int64_t>(1, s.M / (4 * kBK)));
  return (int)sp;
}

static bool tg_layer(const ConvShape& s);

// Workspace: dP (BF16) | split partials (FP32); a tap-GEMM layer's data gradient
// reuses the partials' area (summed by then) for dcol [M][27 Ci] FP32.
size_t conv_ws_bytes(const ConvShape& s) {
  const size_t dp = ((size_t)s.M * s.Co * sizeof(bf16) + 255) / 256 * 256;
  size_t part = (size_t)wgrad_splits(s) * (s.Kp + 1) * s.Co * sizeof(float);
  if (tg_layer(s)) part = std::max(part, (size_t)s.M * 27 * s.Ci * sizeof(float));
  return dp + part + 256;
}

// Column tile of the forward: all Co columns, or fewer (>= 16) when the row tiles
// alone would leave SMs idle (two blocks per SM wanted).
static int fwd_cols(const ConvShape& s) {
  const int64_t tiles = (s.M + kBM - 1) / kBM;
  int bn = s.Co;
  while (bn > 16 && tiles * (s.Co / bn) < 2 * 148) bn /= 2;
  return bn;
}

// Reduction splits of the forward: when the row tiles alone cannot fill the SMs
// (two blocks per SM wanted), all Co columns per block and the reduction split so
// the input is gathered once; at least four 32-element stages per split.
static int fwd_splits(const ConvShape& s) {
  if (conv1_direct(s)) return 1;
  const int64_t tiles = (s.M + kBM - 1) / kBM;
  if (tiles >= 148) return 1;
  const int64_t stages = s.Kp / kBK;
  int64_t sp = std::min<int64_t>((2 * 148 + tiles - 1) / tiles, stages / 4);
  if (sp < 2) return 1;
  const int64_t per = (stages + sp - 1) / sp;
  return (int)((stages + per - 1) / per);
}

// Tap-GEMM forward (conv_tg.cuh): 64 -> 128 channels, whole images of at most 128
// output voxels per tile (128 divisible by the voxels per image).
static bool tg_layer(const ConvShape& s) {
  const int per_img = s.Do * s.Ho * s.Wo;
  return s.Ci == 64 && s.Co == 128 && per_img <= 128 && 128 % per_img == 0;
}
static int64_t tg_tiles(const ConvShape& s) {
  const int nb = 128 / (s.Do * s.Ho * s.Wo);
  return (s.B + nb - 1) / nb;
}
// Taps per split: about one block per SM over the m tiles and the splits.
static int tg_tps(const ConvShape& s) {
  const int64_t sp = std::max<int64_t>(1, std::min<int64_t>(27, 148 / tg_tiles(s)));
  return (int)((27 + sp - 1) / sp);
}
static int tg_splits(const ConvShape& s) { return (27 + tg_tps(s) - 1) / tg_tps(s); }

size_t conv_fwd_ws_bytes(const ConvShape& s) {
  const int sp = fwd_splits(s);
  const size_t split = sp > 1 ? (size_t)sp * s.M * s.Co * sizeof(float) + 256 : 256;
  // a tap-GEMM layer may still take the split path (no tensor map): room for both
  if (tg_layer(s)) return std::max(split, (size_t)tg_splits(s) * s.M * s.Co * sizeof(float) + 256);
  return split;
}

// Footprint kernels (conv_fp.cuh): the layer shapes they are instantiated for.
static bool fp_layer(const ConvShape& s) {
  return (s.Ci == 16 && s.Co == 32) || (s.Ci == 32 && s.Co == 64);
}

// Raises a footprint kernel's dynamic shared-memory limit to its size, once per
// device (a host-side attribute: the first call on a device should come before any
// stream capture).
template <typename Kern>
static cudaError_t fp_smem_once(Kern k, int bytes, std::atomic<bool>* done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < kConvMaxDevices && done[dev].load()) return cudaSuccess;
  e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && dev >= 0 && dev < kConvMaxDevices) done[dev].store(true);
  return e;
}

// Persistent grid of a footprint kernel: as many blocks as the SMs hold at once
// (shared memory bound), never more than the tiles.
static unsigned fp_grid(int64_t tiles, int smem) {
  const int per_sm = std::max(1, 232448 / (smem + 1024));
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)num_sms() * per_sm));
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static std::atomic<void*> fn{nullptr};
  void* f = fn.load();
  if (!f) {
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !f)
      return nullptr;
    fn.store(f);
  }
  return (PFN_cuTensorMapEncodeTiled_v12000)f;
}

// Tensor map of a dense BF16 array of ``rank`` dimensions (innermost first, in
// elements), boxes ``box`` with traversal strides ``estr``, out-of-range elements
// read as zero.  False when the driver refuses it (the caller takes another path).
static bool bf16_tmap(CUtensorMap* m, const void* base, int rank, const cuuint64_t* dims,
                      const cuuint32_t* box, const cuuint32_t* estr,
                      CUtensorMapSwizzle swz = CU_TENSOR_MAP_SWIZZLE_NONE) {
  auto enc = tmap_encoder();
  if (!enc) return false;
  cuuint64_t strides[4];
  cuuint64_t st = 2;
  for (int i = 0; i < rank - 1; ++i) {
    st *= dims[i];
    strides[i] = st;
  }
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (cuuint32_t)rank, const_cast<void*>(base), dims,
             strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// W [27 CI rows][CO] as [tap][ci][co], boxes {8 co, CI, 27}.
static bool weight_tmap(CUtensorMap* m, const ConvShape& s, const bf16* w) {
  const cuuint64_t dims[3] = {(cuuint64_t)s.Co, (cuuint64_t)s.Ci, 27};
  const cuuint32_t box[3] = {8, (cuuint32_t)s.Ci, 27}, estr[3] = {1, 1, 1};
  return bf16_tmap(m, w, 3, dims, box, estr);
}

template <int CI, int CO, int HR>
static int fp_fwd_launch(const ConvShape& s, const bf16* x, const bf16* w, FwdEp ep,
                         cudaStream_t st) {
  CUtensorMap xmap, wmap;
  const cuuint64_t dims[5] = {(cuuint64_t)CI, (cuuint64_t)s.W, (cuuint64_t)s.H, (cuuint64_t)s.D,
                              (cuuint64_t)s.B};
  const cuuint32_t box[5] = {8, 18, HR, 3, 1}, estr[5] = {1, 2, 1, 1, 1};
  if (!bf16_tmap(&xmap, x, 5, dims, box, estr) || !weight_tmap(&wmap, s, w)) return -1;
  static std::atomic<bool> done[kConvMaxDevices];
  auto k = k_conv_fp_fwd<CI, CO, HR>;
  const int smem = FpFwd<CI, CO, HR>::kSmem;
  if (fp_smem_once(k, smem, done) != cudaSuccess) return DM_ERR_CUDA;
  const int64_t tiles = (int64_t)s.B * s.Do * ((s.Ho + 15) / 16) * ((s.Wo + 7) / 8);
  k<<<fp_grid(tiles, smem), kFpThreads, smem, st>>>(xmap, wmap, s, ep, conv_status_ptr());
  count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

// Forward on the footprint kernels: (Ci, Co) = (16, 32) at any size, (32, 64) with
// at most 8 output rows (the 33-row footprint of a 64-channel weight image would not
// fit in shared memory); 16-byte aligned tensors.  Returns false when not taken.
static bool fp_forward(const ConvShape& s, const bf16* x, const bf16* w, const FwdEp& ep,
                       cudaStream_t st, int& rc) {
  if (!fp_layer(s) || !ep.vec || !aligned16(x) || !aligned16(w)) return false;
  if (s.Ci == 16)
    rc = s.Ho > 8 ? fp_fwd_launch<16, 32, 33>(s, x, w, ep, st)
                  : fp_fwd_launch<16, 32, 17>(s, x, w, ep, st);
  else if (s.Ho <= 8)
    rc = fp_fwd_launch<32, 64, 17>(s, x, w, ep, st);
  else
    return false;
  return rc != -1;  // -1: no tensor map, nothing launched
}

template <int CI, int CO>
static int fp_dgrad_launch(const ConvShape& s, const bf16* dp, const bf16* w, float* dx,
                           bf16* dxb, cudaStream_t st) {
  CUtensorMap dmap, wmap;
  const cuuint64_t dims[5] = {(cuuint64_t)CO, (cuuint64_t)s.Wo, (cuuint64_t)s.Ho,
                              (cuuint64_t)s.Do, (cuuint64_t)s.B};
  const cuuint32_t box[5] = {8, 9, 17, 2, 1}, estr[5] = {1, 1, 1, 1, 1};
  if (!bf16_tmap(&dmap, dp, 5, dims, box, estr) || !weight_tmap(&wmap, s, w)) return -1;
  static std::atomic<bool> done[kConvMaxDevices];
  auto k = k_conv_fp_dgrad<CI, CO>;
  const int smem = FpDgrad<CI, CO>::kSmem;
  if (fp_smem_once(k, smem, done) != cudaSuccess) return DM_ERR_CUDA;
  const int nd = (s.D + 1) / 2, nh = (s.H + 1) / 2, nw = (s.W + 1) / 2;
  const int64_t tiles = (int64_t)s.B * nd * ((nh + 15) / 16) * ((nw + 7) / 8);
  k<<<fp_grid(tiles, smem), kFpThreads, smem, st>>>(dmap, wmap, s, dx, dxb, conv_status_ptr());
  count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

static bool tgp_geom(const ConvShape& s, TgGeom& g);

// Data gradient on the per-class tap-GEMM kernel (32 -> 64 channels, even input
// extents).  -1: not taken.
static int tgc_dgrad(const ConvShape& s, const bf16* dp, const bf16* w, float* dx, bf16* dxb,
                     cudaStream_t st) {
  TgGeom g;
  if (s.Ci != 32 || s.Co != 64 || (s.D & 1) || (s.H & 1) || (s.W & 1) || !tgp_geom(s, g) ||
      !aligned16(dp) || !aligned16(w) || !aligned16(dxb ? (void*)dxb : (void*)dx))
    return -1;
  CUtensorMap dmap, wmap;
  const cuuint64_t ddims[5] = {64, (cuuint64_t)s.Wo, (cuuint64_t)s.Ho, (cuuint64_t)s.Do,
                               (cuuint64_t)s.B};
  const cuuint32_t dbox[5] = {64, (cuuint32_t)g.wt, (cuuint32_t)g.ht, (cuuint32_t)g.dt,
                              (cuuint32_t)g.nbt};
  const cuuint32_t destr[5] = {1, 1, 1, 1, 1};
  const cuuint64_t wdims[2] = {64, (cuuint64_t)(27 * 32)};
  const cuuint32_t wbox[2] = {64, 32}, westr[2] = {1, 1};
  if (!bf16_tmap(&dmap, dp, 5, ddims, dbox, destr, CU_TENSOR_MAP_SWIZZLE_128B) ||
      !bf16_tmap(&wmap, w, 2, wdims, wbox, westr, CU_TENSOR_MAP_SWIZZLE_128B))
    return -1;
  using F = TgcDgrad<32, 64>;
  static std::atomic<bool> done[kConvMaxDevices];
  auto k = k_conv_tgc_dgrad<32, 64>;
  if (fp_smem_once(k, F::kSmem, done) != cudaSuccess) return DM_ERR_CUDA;
  const int64_t tiles = 8 * (int64_t)g.nbk * g.nd * g.nh;
  const int per_sm = std::max(1, std::min(232448 / (F::kSmem + 1024), 512 / F::kCols));
  const unsigned grid =
      (unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)per_sm * num_sms()));
  k<<<grid, 160, F::kSmem, st>>>(dmap, wmap, s, g, dx, dxb, conv_status_ptr());
  count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

// Data gradient on the footprint kernel (all eight parity classes per tile).
static bool fp_dgrad(const ConvShape& s, const bf16* dp, const bf16* w, float* dx, bf16* dxb,
                     cudaStream_t st, int& rc) {
  if (!fp_layer(s) || !aligned16(dp) || !aligned16(w) || !aligned16(dxb ? (void*)dxb : (void*)dx))
    return false;
  if (s.Ci == 32) {
    rc = tgc_dgrad(s, dp, w, dx, dxb, st);
    if (rc != -1) return true;
  }
  rc = s.Ci == 16 ? fp_dgrad_launch<16, 32>(s, dp, w, dx, dxb, st)
                  : fp_dgrad_launch<32, 64>(s, dp, w, dx, dxb, st);
  return rc != -1;
}

template <int CI, int CO>
static cudaError_t fp_wgrad_launch(const ConvShape& s, const bf16* x, const bf16* dp, float* part,
                                   int splits, int& used, cudaStream_t st) {
  static std::atomic<bool> done[kConvMaxDevices];
  auto k = k_conv_fp_wgrad<CI, CO>;
  const int smem = FpWgrad<CI, CO>::kSmem;
  cudaError_t e = fp_smem_once(k, smem, done);
  if (e != cudaSuccess) return e;
  const int64_t tiles = (int64_t)s.B * s.Do * ((s.Ho + 15) / 16) * ((s.Wo + 7) / 8);
  const int64_t per = (tiles + splits - 1) / splits;
  used = (int)((tiles + per - 1) / per);
  k<<<dim3((unsigned)used, 3), kFpThreads, smem, st>>>(x, s, dp, (int)per, part,
                                                       conv_status_ptr());
  count_launches(1);
  return cudaGetLastError();
}

// Weight + bias gradient partials on the footprint kernel: blocks (split, kd), at most
// as many splits as the workspace holds, about one wave of blocks (three per SM for
// Ci = 16, two for Ci = 32) and at least eight forward tiles per split.
static bool fp_wgrad(const ConvShape& s, const bf16* x, const bf16* dp, float* part, int& used,
                     cudaStream_t st, int& rc) {
  if (!fp_layer(s) || !aligned16(x) || !aligned16(dp) || !aligned16(part)) return false;
  const int64_t tiles = (int64_t)s.B * s.Do * ((s.Ho + 15) / 16) * ((s.Wo + 7) / 8);
  const int64_t wave = (int64_t)148 * (s.Ci == 16 ? 3 : 2) / 3;
  const int splits = (int)std::max<int64_t>(
      1, std::min<int64_t>({wave, tiles / 8, (int64_t)wgrad_splits(s)}));
  const cudaError_t e = s.Ci == 16 ? fp_wgrad_launch<16, 32>(s, x, dp, part, splits, used, st)
                                   : fp_wgrad_launch<32, 64>(s, x, dp, part, splits, used, st);
  rc = e == cudaSuccess ? DM_OK : DM_ERR_CUDA;
  return true;
}

// Single-channel layer on the space-to-depth kernels (conv_s2d.cuh): W even (each
// block's column pairs are 4-byte words), x 4-byte aligned, outputs 16-byte aligned.
static bool s2d_layer(const ConvShape& s, const bf16* x) {
  return conv1_direct(s) && (s.W & 1) == 0 && ((uintptr_t)x & 3u) == 0;
}

template <int CO>
static cudaError_t s2d_fwd_launch(const ConvShape& s, const bf16* x, const bf16* w,
                                  const float* bias, float* pre, bf16* act, cudaStream_t st) {
  static std::atomic<bool> done[kConvMaxDevices];
  auto k = k_conv_s2d_fwd_ws<CO>;
  const int smem = S2dFwdWs<CO>::kSmem;
  cudaError_t e = fp_smem_once(k, smem, done);
  if (e != cudaSuccess) return e;
  const int64_t tiles = (int64_t)s.B * s.Do * ((s.Ho + 15) / 16) * ((s.Wo + 7) / 8);
  // one wave: the blocks of 256 threads the SMs' registers hold at once
  cudaFuncAttributes fa;
  int per_sm = 4;
  if (cudaFuncGetAttributes(&fa, k) == cudaSuccess && fa.numRegs > 0)
    per_sm = std::max(1, std::min(8, 65536 / (256 * ((fa.numRegs + 7) / 8 * 8))));
  const unsigned grid =
      (unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)per_sm * num_sms()));
  k<<<grid, 256, smem, st>>>(x, s, w, bias, pre, act, conv_status_ptr());
  count_launches(1);
  return cudaGetLastError();
}

template <int CO, bool VEC>
static cudaError_t s2d_wgrad_launch(const ConvShape& s, const bf16* x, const bf16* dp,
                                    float* part, int splits, int& used, cudaStream_t st) {
  static std::atomic<bool> done[kConvMaxDevices];
  auto k = k_conv_s2d_wgrad<CO, VEC>;
  const int smem = S2dWgrad<CO>::kSmem;
  cudaError_t e = fp_smem_once(k, smem, done);
  if (e != cudaSuccess) return e;
  const int64_t tiles = (int64_t)s.B * s.Do * ((s.Ho + 15) / 16) * ((s.Wo + 7) / 8);
  const int64_t per = (tiles + splits - 1) / splits;
  used = (int)((tiles + per - 1) / per);
  k<<<(unsigned)used, 256, smem, st>>>(x, s, dp, (int)per, part, conv_status_ptr());
  count_launches(1);
  return cudaGetLastError();
}

// Forward of a tap-GEMM layer: the tap GEMM's partials into the workspace, their
// fixed-order sum with the bias and GELU.  -1: not taken (no tensor map).
static int tg_forward(const ConvShape& s, const bf16* x, const bf16* w, const float* bias,
                      float* pre, bf16* act, void* ws, cudaStream_t st) {
  float* part = (float*)ws;
  const int K = 27 * s.Ci, nb = 128 / (s.Do * s.Ho * s.Wo);
  CUtensorMap xmap, wmap;
  {
    const cuuint64_t dims[5] = {(cuuint64_t)s.Ci, (cuuint64_t)s.W, (cuuint64_t)s.H,
                                (cuuint64_t)s.D, (cuuint64_t)s.B};
    const cuuint32_t box[5] = {64, (cuuint32_t)(2 * s.Wo), (cuuint32_t)(2 * s.Ho),
                               (cuuint32_t)(2 * s.Do), (cuuint32_t)nb};
    const cuuint32_t estr[5] = {1, 2, 2, 2, 1};
    const cuuint64_t wdims[2] = {(cuuint64_t)s.Co, (cuuint64_t)K};
    const cuuint32_t wbox[2] = {64, 64}, westr[2] = {1, 1};
    if (!bf16_tmap(&xmap, x, 5, dims, box, estr, CU_TENSOR_MAP_SWIZZLE_128B) ||
        !bf16_tmap(&wmap, w, 2, wdims, wbox, westr, CU_TENSOR_MAP_SWIZZLE_128B))
      return -1;
  }
  static std::atomic<bool> done[kConvMaxDevices];
  const int smem = 1024 + kTgStages * kTgStageBytes + 128;
  if (fp_smem_once(k_conv_tg_fwd, smem, done) != cudaSuccess) return DM_ERR_CUDA;
  const int tps = tg_tps(s), sp = tg_splits(s);
  k_conv_tg_fwd<<<dim3((unsigned)tg_tiles(s), (unsigned)sp), 128, smem, st>>>(
      xmap, wmap, s, tps, part, conv_status_ptr());
  const int64_t n = s.M * s.Co;
  k_fwd_reduce<<<(unsigned)std::min<int64_t>((n / 4 + 255) / 256, 148 * 16), 256, 0, st>>>(
      part, sp, n, s.Co, bias, pre, act);
  count_launches(2);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

static bool tgp_geom(const ConvShape& s, TgGeom& g);

// Weight + bias gradient on the tap-GEMM kernel: blocks (tap group or bias, split
// over m tiles), partials into part, ``used`` splits.  -1: not taken.
template <int CI, int CO>
static int tg_wgrad_t(const ConvShape& s, const TgGeom& g, const bf16* x, const bf16* dp,
                      float* part, int& used, cudaStream_t st) {
  CUtensorMap xmap, dmap;
  const cuuint64_t dims[5] = {(cuuint64_t)CI, (cuuint64_t)s.W, (cuuint64_t)s.H, (cuuint64_t)s.D,
                              (cuuint64_t)s.B};
  const cuuint32_t box[5] = {CI, (cuuint32_t)(2 * g.wt), (cuuint32_t)(2 * g.ht),
                             (cuuint32_t)(2 * g.dt), (cuuint32_t)g.nbt};
  const cuuint32_t estr[5] = {1, 2, 2, 2, 1};
  const cuuint64_t ddims[2] = {(cuuint64_t)CO, (cuuint64_t)s.M};
  const cuuint32_t dbox[2] = {64, 128}, destr[2] = {1, 1};
  const CUtensorMapSwizzle xs = CI == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B;
  if (!bf16_tmap(&xmap, x, 5, dims, box, estr, xs) ||
      !bf16_tmap(&dmap, dp, 2, ddims, dbox, destr, CU_TENSOR_MAP_SWIZZLE_128B))
    return -1;
  using F = TgWgrad<CI, CO>;
  static std::atomic<bool> done[kConvMaxDevices];
  auto k = k_conv_tg_wgrad<CI, CO>;
  if (fp_smem_once(k, F::kSmem, done) != cudaSuccess) return DM_ERR_CUDA;
  const int64_t mtiles = (int64_t)g.nbk * g.nd * g.nh;
  // about one wave: blocks per SM from shared memory, over the tap groups + bias
  const int per_sm = std::max(1, 232448 / (F::kSmem + 1024));
  const int64_t cap = std::max<int64_t>(1, (int64_t)num_sms() * per_sm / (F::kGroups + 1));
  const int sp = (int)std::max<int64_t>(1, std::min<int64_t>({cap, mtiles, (int64_t)wgrad_splits(s)}));
  const int64_t per = (mtiles + sp - 1) / sp;
  used = (int)((mtiles + per - 1) / per);
  k<<<dim3(F::kGroups + 1, (unsigned)used), 128, F::kSmem, st>>>(xmap, dmap, s, g, (int)per, part,
                                                                   conv_status_ptr());
  count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

static int tg_wgrad(const ConvShape& s, const bf16* x, const bf16* dp, float* part, int& used,
                    cudaStream_t st) {
  TgGeom g;
  if (!tgp_geom(s, g) || !aligned16(x) || !aligned16(dp) || !aligned16(part)) return -1;
  if (s.Ci == 64 && s.Co == 128) return tg_wgrad_t<64, 128>(s, g, x, dp, part, used, st);
  if (s.Ci == 32 && s.Co == 64) return tg_wgrad_t<32, 64>(s, g, x, dp, part, used, st);
  return -1;
}

// Data gradient of a tap-GEMM layer: dcol = dP W^T per (m tile, 4 taps) into the
// workspace, then the fixed-order col2im gather into dx.  -1: not taken.
static int tg_dgrad(const ConvShape& s, const bf16* dp, const bf16* w, float* dcol, float* dx,
                    bf16* dxb, cudaStream_t st) {
  CUtensorMap dmap, wmap;
  const cuuint64_t ddims[2] = {(cuuint64_t)s.Co, (cuuint64_t)s.M};
  const cuuint64_t wdims[2] = {(cuuint64_t)s.Co, (cuuint64_t)(27 * s.Ci)};
  const cuuint32_t dbox[2] = {64, 128}, wbox[2] = {64, 256}, estr[2] = {1, 1};
  if (!bf16_tmap(&dmap, dp, 2, ddims, dbox, estr, CU_TENSOR_MAP_SWIZZLE_128B) ||
      !bf16_tmap(&wmap, w, 2, wdims, wbox, estr, CU_TENSOR_MAP_SWIZZLE_128B))
    return -1;
  static std::atomic<bool> done[kConvMaxDevices];
  if (fp_smem_once(k_conv_tg_dgrad, kTgDgradSmem, done) != cudaSuccess) return DM_ERR_CUDA;
  k_conv_tg_dgrad<<<dim3((unsigned)((s.M + 127) / 128), (27 * s.Ci + 255) / 256), 128,
                    kTgDgradSmem, st>>>(dmap, wmap, s, dcol, conv_status_ptr());
  const int64_t n = (int64_t)s.B * s.D * s.H * s.W * 16;
  k_conv_col2im<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16), 256, 0, st>>>(
      dcol, s, dx, dxb);
  count_launches(2);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

// Tile geometry of the persistent tap GEMM (conv_tg.cuh): 128 output voxels as
// Wt = Wo voxels x Ht rows x Dt planes x nbt images.  False when Wo does not divide
// 128 or the rows / planes do not fill a tile exactly.
static bool tgp_geom(const ConvShape& s, TgGeom& g) {
  if (s.Wo > 128 || 128 % s.Wo) return false;
  g.wt = s.Wo;
  const int r = 128 / s.Wo;
  g.ht = r; g.nh = (s.Ho + r - 1) / r; g.dt = 1; g.nd = s.Do; g.nbt = 1;
  if (s.Ho < r) {
    if (r % s.Ho) return false;
    g.ht = s.Ho; g.nh = 1;
    const int r2 = r / s.Ho;
    g.dt = r2; g.nd = (s.Do + r2 - 1) / r2;
    if (s.Do < r2) {
      if (r2 % s.Do) return false;
      g.dt = s.Do; g.nd = 1; g.nbt = r2 / s.Do;
    }
  }
  g.nbk = (s.B + g.nbt - 1) / g.nbt;
  return g.wt * g.ht * g.dt * g.nbt == 128;
}

template <int CI, int CO>
static int tgp_fwd_launch(const ConvShape& s, const TgGeom& g, const bf16* x, const bf16* w,
                          const FwdEp& ep, cudaStream_t st) {
  CUtensorMap xmap, wmap;
  const cuuint64_t dims[5] = {(cuuint64_t)CI, (cuuint64_t)s.W, (cuuint64_t)s.H, (cuuint64_t)s.D,
                              (cuuint64_t)s.B};
  const cuuint32_t box[5] = {CI, (cuuint32_t)(2 * g.wt), (cuuint32_t)(2 * g.ht),
                             (cuuint32_t)(2 * g.dt), (cuuint32_t)g.nbt};
  const cuuint32_t estr[5] = {1, 2, 2, 2, 1};
  const cuuint64_t wdims[2] = {(cuuint64_t)CO, (cuuint64_t)(27 * CI)};
  const cuuint32_t wbox[2] = {CO, CI}, westr[2] = {1, 1};
  const CUtensorMapSwizzle xs = CI == 16 ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_64B;
  const CUtensorMapSwizzle wsz = CO == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B;
  if (!bf16_tmap(&xmap, x, 5, dims, box, estr, xs) || !bf16_tmap(&wmap, w, 2, wdims, wbox, westr, wsz))
    return -1;
  using F = TgpFwd<CI, CO>;
  static std::atomic<bool> done[kConvMaxDevices];
  auto k = k_conv_tgp_fwd<CI, CO>;
  if (fp_smem_once(k, F::kSmem, done) != cudaSuccess) return DM_ERR_CUDA;
  const int64_t tiles = (int64_t)g.nbk * g.nd * g.nh;
  const int per_sm = std::max(1, std::min({232448 / (F::kSmem + 1024), 512 / F::kCols, 12}));
  const unsigned grid =
      (unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)per_sm * num_sms()));
  k<<<grid, 160, F::kSmem, st>>>(xmap, wmap, s, g, ep, conv_status_ptr());
  count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

int launch_conv_forward(const ConvShape& s, const bf16* x, const bf16* w, const float* bias,
                        float* pre, bf16* act, cudaStream_t st, void* ws = nullptr,
                        size_t ws_bytes = 0) {
  {
    TgGeom g;
    const FwdEp ep{bias, pre, act, s.Co, 0, aligned16(pre) && aligned16(act)};
    // 32 -> 64 channels: a tap's 64-byte rows keep the boxes large enough for the TMA
    // engine (the 16-channel layer's 32-byte rows made its 27 boxes per tile slower
    // than the footprint kernel: 68 against 60 us at batch 64, 32^3 in)
    if (s.Ci == 32 && s.Co == 64 && tgp_geom(s, g) && ep.vec && aligned16(x) && aligned16(w)) {
      const int rc = tgp_fwd_launch<32, 64>(s, g, x, w, ep, st);
      if (rc != -1) return rc;
    }
  }
  if (tg_layer(s) && ws && ws_bytes >= conv_fwd_ws_bytes(s) && aligned16(x) && aligned16(w) &&
      aligned16(pre) && aligned16(act) && aligned16(ws)) {
    const int rc = tg_forward(s, x, w, bias, pre, act, ws, st);
    if (rc != -1) return rc;
  }
  if (s2d_layer(s, x) && s.W % 8 == 0 && aligned16(x) && aligned16(pre) && aligned16(act)) {
    const cudaError_t e = s.Co == 16 ? s2d_fwd_launch<16>(s, x, w, bias, pre, act, st)
                                     : s2d_fwd_launch<32>(s, x, w, bias, pre, act, st);
    return e == cudaSuccess ? DM_OK : DM_ERR_CUDA;
  }
  {
    int rc = DM_OK;
    if (fp_forward(s, x, w, FwdEp{bias, pre, act, s.Co, 0, aligned16(pre) && aligned16(act)}, st,
                   rc))
      return rc;
  }
  const int sp = fwd_splits(s);
  if (sp > 1 && ws && ws_bytes >= conv_fwd_ws_bytes(s) && aligned16(ws) && aligned16(pre) &&
      aligned16(act) && s.Co % 16 == 0) {
    const int64_t stages = s.Kp / kBK;
    const int64_t per = (stages + sp - 1) / sp * kBK;
    float* part = (float*)ws;
    gemm_launch(s.Co, FwdA{x, s, s.Ci % 8 == 0 && aligned16(x)}, WeightB{w, s.Co, 0},
                FwdSplitEp{part, s.M * s.Co, s.Co, 0}, s.M, s.Kp, per, sp, 1, st);
    const int64_t n = s.M * s.Co;
    k_fwd_reduce<<<(unsigned)std::min<int64_t>((n / 4 + 255) / 256, 148 * 16), 256, 0, st>>>(
        part, sp, n, s.Co, bias, pre, act);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
  }
  if (conv1_direct(s) && aligned16(pre) && aligned16(act)) {
    const unsigned g = (unsigned)conv1_tiles_host(s);
    if (s.Co == 16)
      k_conv1_fwd<16><<<g, 256, 0, st>>>(x, s, w, bias, pre, act);
    else
      k_conv1_fwd<32><<<g, 256, 0, st>>>(x, s, w, bias, pre, act);
    count_launches(1);
    return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
  }
  const int bn = fwd_cols(s);
  gemm_launch(bn, FwdA{x, s, s.Ci % 8 == 0 && aligned16(x)}, WeightB{w, s.Co, 0},
              FwdEp{bias, pre, act, s.Co, 0, aligned16(pre) && aligned16(act)}, s.M, s.Kp, s.Kp,
              1, s.Co / bn, st);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

template <class TG>
static void gelu_back(const float* pre, const TG* dact, bf16* dp, int64_t nout, cudaStream_t st) {
  if (aligned16(pre) && aligned16(dact) && aligned16(dp))  // nout: a multiple of 16
    k_gelu_back<true, TG><<<(unsigned)std::min<int64_t>((nout / 4 + 255) / 256, 148 * 16), 256,
                            0, st>>>(pre, dact, dp, nout);
  else
    k_gelu_back<false, TG><<<(unsigned)std::min<int64_t>((nout + 255) / 256, 148 * 16), 256, 0,
                             st>>>(pre, dact, dp, nout);
}

int launch_conv_backward(const ConvShape& s, const bf16* x, const bf16* w, const float* pre,
                         const float* dact, const bf16* dact_b, float* dx, bf16* dx_b, float* dw,
                         float* db, void* ws, cudaStream_t st) {
  char* base = (char*)ws;
  bf16* dp = (bf16*)base;
  float* part = (float*)(base + ((size_t)s.M * s.Co * sizeof(bf16) + 255) / 256 * 256);
  const int64_t nout = s.M * s.Co;
  if (dact_b)
    gelu_back(pre, dact_b, dp, nout, st);
  else
    gelu_back(pre, dact, dp, nout, st);
  count_launches(1);
  // weight and bias gradients: rows = Kp + 1 (the last row of A^T is ones), the
  // reduction over m split across blockIdx.y
  const int splits = wgrad_splits(s);
  int used;
  if (s2d_layer(s, x) && aligned16(dp) && aligned16(part)) {
    // one wave of blocks (three per SM), at least eight tiles per block
    const int64_t tiles = (int64_t)s.B * s.Do * ((s.Ho + 15) / 16) * ((s.Wo + 7) / 8);
    const int sp = (int)std::max<int64_t>(
        1, std::min<int64_t>({(int64_t)3 * num_sms(), tiles / 8, (int64_t)splits}));
    const bool vec = s.W % 8 == 0 && aligned16(x);
    const cudaError_t e =
        s.Co == 16 ? (vec ? s2d_wgrad_launch<16, true>(s, x, dp, part, sp, used, st)
                          : s2d_wgrad_launch<16, false>(s, x, dp, part, sp, used, st))
                   : (vec ? s2d_wgrad_launch<32, true>(s, x, dp, part, sp, used, st)
                          : s2d_wgrad_launch<32, false>(s, x, dp, part, sp, used, st));
    if (e != cudaSuccess) return DM_ERR_CUDA;
  } else if (conv1_direct(s)) {
    used = (int)std::max<int64_t>(1, std::min<int64_t>(splits, conv1_tiles_host(s)));
    if (s.Co == 16)
      k_conv1_wgrad<16><<<used, 256, 0, st>>>(x, s, dp, part);
    else
      k_conv1_wgrad<32><<<used, 256, 0, st>>>(x, s, dp, part);
    count_launches(1);
  } else if (int trc = tg_wgrad(s, x, dp, part, used, st); trc != -1) {
    if (trc != DM_OK) return trc;
  } else if (int rc = DM_OK; fp_wgrad(s, x, dp, part, used, st, rc)) {
    if (rc != DM_OK) return rc;
  } else {
    const int64_t per = ((s.M + splits - 1) / splits + kBK - 1) / kBK * kBK;
    used = (int)((s.M + per - 1) / per);
    gemm_launch(s.Co, WgradA{x, s, s.Ci % 8 == 0 && aligned16(x)},
                DpreB{dp, s.Co, aligned16(dp)},
                WgradEp{part, (int64_t)(s.Kp + 1) * s.Co, s.Co}, (int64_t)s.Kp + 1, s.M, per,
                used, 1, st);
  }
  const int64_t nw = (int64_t)s.Kp * s.Co;
  k_sum_splits<<<(unsigned)((nw + s.Co + 31) / 32), dim3(32, 8), 0, st>>>(part, used, nw, s.Co,
                                                                          dw, db);
  count_launches(1);
  // data gradient: the eight parity classes of the input voxels in one launch
  if (dx || dx_b) {
    int rc = DM_OK;
    if (tg_layer(s) && aligned16(dp) && aligned16(w) && aligned16(part) &&
        aligned16(dx_b ? (void*)dx_b : (void*)dx)) {
      rc = tg_dgrad(s, dp, w, part, dx, dx_b, st);
      if (rc != -1) return rc;
    }
    if (fp_dgrad(s, dp, w, dx, dx_b, st, rc)) return rc;
    ClsSet set;
    int64_t max_rows = 0, max_red = 0;
    const int dims[3] = {s.D, s.H, s.W};
    // z = 7 - parity bits: the class with the most taps (all odd) first, so the
    // longest blocks are not the last to start
    for (int z = 0; z < 8; ++z) {
      const int cls = 7 - z;
      Cls& c = set.c[z];
      c.T = 1;
      bool empty = false;
      for (int a = 0; a < 3; ++a) {
        c.p[a] = (cls >> (2 - a)) & 1;
        c.n[a] = (dims[a] - c.p[a] + 1) / 2;
        c.nt[a] = c.p[a] == 0 ? 1 : 2;
        c.T *= c.nt[a];
        if (c.n[a] <= 0) empty = true;
      }
      c.rows = empty ? 0 : (int64_t)s.B * c.n[0] * c.n[1] * c.n[2];
      c.red = ((int64_t)c.T * s.Co + kBK - 1) / kBK * kBK;
      max_rows = std::max(max_rows, c.rows);
      max_red = std::max(max_red, c.red);
    }
    const bool dvec = (dx_b ? aligned16(dx_b) : aligned16(dx)) && s.Ci % 16 == 0;
    gemm_launch(pad_cols(s.Ci), DgradA{dp, s, set, Cls{}, aligned16(dp)},
                DgradB{w, s, set, Cls{}, aligned16(w)},
                DgradEp{dx_b ? nullptr : dx, dx_b, s, set, Cls{}, dvec},
                max_rows, max_red, max_red, 1, 8, st);
  }
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

}  // namespace dm

// ---------------------------------------------------------------------------
extern "C" {

size_t dm_conv3d_s2_workspace_size(int B, int D, int H, int W, int Ci, int Co) {
  dm::ConvShape s;
  if (!dm::conv_shape(B, D, H, W, Ci, Co, s)) return 0;
  return dm::conv_ws_bytes(s);
}

int dm_conv3d_s2_forward(const uint16_t* x, int B, int D, int H, int W, int Ci, const uint16_t* w,
                         const float* bias, int Co, float* pre, uint16_t* act,
                         dm_stream_t stream) {
  dm::ConvShape s;
  if (!dm::conv_shape(B, D, H, W, Ci, Co, s)) return DM_ERR_INVALID_ARG;
  if (!x || !w || !pre || !act) return DM_ERR_INVALID_ARG;
  return dm::launch_conv_forward(s, (const dm::bf16*)x, (const dm::bf16*)w, bias, pre,
                                 (dm::bf16*)act, (cudaStream_t)stream);
}

size_t dm_conv3d_s2_forward_workspace_size(int B, int D, int H, int W, int Ci, int Co) {
  dm::ConvShape s;
  if (!dm::conv_shape(B, D, H, W, Ci, Co, s)) return 0;
  return dm::conv_fwd_ws_bytes(s);
}

int dm_conv3d_s2_forward_ws(const uint16_t* x, int B, int D, int H, int W, int Ci,
                            const uint16_t* w, const float* bias, int Co, float* pre,
                            uint16_t* act, void* workspace, size_t ws_bytes, dm_stream_t stream) {
  dm::ConvShape s;
  if (!dm::conv_shape(B, D, H, W, Ci, Co, s)) return DM_ERR_INVALID_ARG;
  if (!x || !w || !pre || !act || !workspace) return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm::conv_fwd_ws_bytes(s)) return DM_ERR_WORKSPACE;
  return dm::launch_conv_forward(s, (const dm::bf16*)x, (const dm::bf16*)w, bias, pre,
                                 (dm::bf16*)act, (cudaStream_t)stream, workspace, ws_bytes);
}

int dm_conv3d_s2_device_error(int* out_flags, dm_stream_t stream) {
  if (!out_flags) return DM_ERR_INVALID_ARG;
  int* p = dm::conv_status_ptr();
  if (!p) return DM_ERR_CUDA;
  int v = 0;
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemcpyAsync(&v, p, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return DM_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return DM_ERR_CUDA;
  if (cudaMemsetAsync(p, 0, sizeof(int), st) != cudaSuccess) return DM_ERR_CUDA;
  *out_flags = v;
  return DM_OK;
}

int dm_conv3d_s2_backward(const uint16_t* x, int B, int D, int H, int W, int Ci,
                          const uint16_t* w, int Co, const float* pre, const float* dact,
                          float* dx, float* dw, float* db, void* workspace, size_t ws_bytes,
                          dm_stream_t stream) {
  dm::ConvShape s;
  if (!dm::conv_shape(B, D, H, W, Ci, Co, s)) return DM_ERR_INVALID_ARG;
  if (!x || !w || !pre || !dact || !dw || !db || !workspace) return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm::conv_ws_bytes(s)) return DM_ERR_WORKSPACE;
  return dm::launch_conv_backward(s, (const dm::bf16*)x, (const dm::bf16*)w, pre, dact, nullptr,
                                  dx, nullptr, dw, db, workspace, (cudaStream_t)stream);
}

int dm_conv3d_s2_backward_bf16(const uint16_t* x, int B, int D, int H, int W, int Ci,
                               const uint16_t* w, int Co, const float* pre, const uint16_t* dact,
                               uint16_t* dx, float* dw, float* db, void* workspace,
                               size_t ws_bytes, dm_stream_t stream) {
  dm::ConvShape s;
  if (!dm::conv_shape(B, D, H, W, Ci, Co, s)) return DM_ERR_INVALID_ARG;
  if (!x || !w || !pre || !dact || !dw || !db || !workspace) return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm::conv_ws_bytes(s)) return DM_ERR_WORKSPACE;
  return dm::launch_conv_backward(s, (const dm::bf16*)x, (const dm::bf16*)w, pre, nullptr,
                                  (const dm::bf16*)dact, nullptr, (dm::bf16*)dx, dw, db,
                                  workspace, (cudaStream_t)stream);
}

}  // extern "C"
