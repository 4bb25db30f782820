// Render + image loss + adjoint for a spectrum that is zero outside the narrow
// band: separable inverse / forward DFTs pruned to the band's bounding box.
//
// The reference renders with torch.fft.ifftn of the dense spectrum
// (render.py:177-180) and its fitting loop back-propagates through it with a
// dense fftn.  The spectrum S = ft * OTF is non-zero only on the band, whose
// voxels lie in the index box [lo_d, lo_d + ext_d) (at 200^3 with the
// anisotropic PSF: 44 x 44 x 22 of 200^3).  With w_d = e^{2 pi i / n_d}:
//
//   T1[x0][j1][j2] = sum_j0 S[lo0+j0][lo1+j1][lo2+j2] w0^{(lo0+j0) x0}     (axis 0)
//   T2[x0][x1][j2] = sum_j1 T1[x0][j1][j2] w1^{(lo1+j1) x1}                (axis 1)
//   z[x0][x1][x2]  = 1/N sum_j2 T2[x0][x1][j2] w2^{(lo2+j2) x2}            (axis 2, lines)
//
// which is ifftn(S) exactly (the DFT is separable; only zero terms are left out).
// The axis-2 pass is the only one over the whole grid.  It also forms |z| and
// its min / max.  A second line pass forms the normalised image, the loss and
// g = dL/dz (normalize_tensor, render.py:5-6, and the loss of the fitting loop),
// and contracts each line with conj(w2) at once; two small pruned passes and a
// gather at the band voxels then give G = fftn(dL/dz) on the band -- the
// cotangent the meshFT adjoint takes.  Full-grid traffic per step: z written
// once and read once, the target read once.
//
// Every sum has a fixed order (no atomics on values): results are bitwise
// reproducible.  The min / max gradient is shared evenly by tied voxels as
// torch's min/max backward does (a single voxel is the common case, added in
// the gather; several are folded into the line contractions by k_bb_ties).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

#include "band_internal.h"
#include "dm_common.cuh"
#include "meshft_internal.h"

namespace dm {
namespace {

constexpr int kLines = 32;         // grid lines (x0, x1) per CTA of the line passes
constexpr int kLineThreads = 256;  // 8 warps; warp w owns lines 4w..4w+3 (z pass)
constexpr int kMaxExt2 = 64;       // band extent along axis 2 served by the line passes
constexpr int kGemmThreads = 256;
constexpr int kSmemLimit = 220 * 1024;

struct BBShape {
  int32_t n[3];    // box shape
  int32_t lo[3];   // band box lower index per axis
  int32_t ext[3];  // band box extent per axis
  int32_t ldj;     // row length of the transposed axis-2 table: ext2 rounded up to 8
  int32_t zc;      // z pass: columns per thread (column block of 32 zc)
  int32_t ldw2;    // row length of the axis-2 table: n2 rounded up to whole column blocks
  int32_t q1split; // K split of the axis-1 forward contraction (partials summed by the next)
  int32_t q1chunk; // positions x1 per split (a multiple of 16)
  int64_t nlines;  // n0 * n1
  int64_t nvox;
};

// min / max of |z| with the first flat index of each and the number of ties
// (box sizes stay below 2^31 voxels)
struct MMC {
  float mn, mx;
  int32_t imn, imx;
  int32_t cmn, cmx;
};

struct LP {
  double loss, dmn, dmx;
};

// Per-call state in the workspace header.
struct BBHdr {
  int err;
  int ties_full;      // several voxels tie at the min or max: k_bb_ties folds them in
  unsigned int done[2];  // CTAs finished in the z / gradient pass (last one reduces)
  float mn, mx;
  int64_t imn, imx, cmn, cmx;
  float add_mn, add_mx;  // d loss / d min (max) per tied voxel
  double fin[3];         // loss, d loss / d min, d loss / d max
};

__device__ __forceinline__ float cabs2(float2 z) { return sqrtf(fmaf(z.x, z.x, z.y * z.y)); }

// acc += a b (complex) on the paired FP32 path: two FFMA2, each rounding once per
// component in the order re: + a.x b.x, - a.y b.y; im: + a.x b.y, + a.y b.x (the
// same results as four scalar FMAs in that order).  In unrolled register tiles the
// broadcast pairs (a.x, a.x), (a.y, a.y) and the swapped (-b.y, b.x) are shared.
__device__ __forceinline__ float2 cmac(float2 acc, float2 a, float2 b) {
  acc = __ffma2_rn(make_float2(a.x, a.x), b, acc);
  acc = __ffma2_rn(make_float2(a.y, a.y), make_float2(-b.y, b.x), acc);
  return acc;
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// e^{2 pi i (k x mod n) / n}, exact index arithmetic, double-precision angle.
__device__ __forceinline__ float2 unit_root(int32_t k, int32_t x, int32_t n) {
  const int64_t r = ((int64_t)k * (int64_t)x) % (int64_t)n;
  double s, c;
  sincospi(2.0 * (double)r / (double)n, &s, &c);
  return make_float2((float)c, (float)s);
}

__device__ __forceinline__ void mmc_add(MMC& r, float a, int32_t i) {
  if (a < r.mn) {
    r.mn = a;
    r.imn = i;
    r.cmn = 1;
  } else if (a == r.mn) {
    r.cmn += 1;
    if (i < r.imn) r.imn = i;
  }
  if (a > r.mx) {
    r.mx = a;
    r.imx = i;
    r.cmx = 1;
  } else if (a == r.mx) {
    r.cmx += 1;
    if (i < r.imx) r.imx = i;
  }
}

__device__ __forceinline__ void mmc_merge(MMC& r, const MMC& o) {
  if (o.mn < r.mn) {
    r.mn = o.mn;
    r.imn = o.imn;
    r.cmn = o.cmn;
  } else if (o.mn == r.mn) {
    r.cmn += o.cmn;
    r.imn = min(r.imn, o.imn);
  }
  if (o.mx > r.mx) {
    r.mx = o.mx;
    r.imx = o.imx;
    r.cmx = o.cmx;
  } else if (o.mx == r.mx) {
    r.cmx += o.cmx;
    r.imx = min(r.imx, o.imx);
  }
}

__device__ __forceinline__ MMC mmc_shfl(const MMC& r, int o) {
  MMC q;
  q.mn = __shfl_down_sync(0xffffffffu, r.mn, o);
  q.mx = __shfl_down_sync(0xffffffffu, r.mx, o);
  q.imn = __shfl_down_sync(0xffffffffu, r.imn, o);
  q.imx = __shfl_down_sync(0xffffffffu, r.imx, o);
  q.cmn = __shfl_down_sync(0xffffffffu, r.cmn, o);
  q.cmx = __shfl_down_sync(0xffffffffu, r.cmx, o);
  return q;
}

// ---------------------------------------------------------------------------
// Root tables: W_d[j][x] = w_d^{(lo_d + j) x} (rows j < ext_d, columns x < n_d;
// the axis-2 rows padded with zeros to ldw2), and the conjugate axis-2 table
// transposed, W2T[x][j] (rows padded to ldj).  Also clears the CTA counters.

__global__ void k_bb_tables(BBShape s, float2* __restrict__ w0, float2* __restrict__ w1,
                            float2* __restrict__ w2, float2* __restrict__ w2t, BBHdr* hdr) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    hdr->done[0] = 0u;
    hdr->done[1] = 0u;
  }
  const int64_t e0 = (int64_t)s.ext[0] * s.n[0];
  const int64_t e1 = (int64_t)s.ext[1] * s.n[1];
  const int64_t e2 = (int64_t)s.ext[2] * s.ldw2;
  const int64_t e3 = (int64_t)s.n[2] * s.ldj;
  const int64_t tot = e0 + e1 + e2 + e3;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < tot;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (i < e0) {
      const int j = (int)(i / s.n[0]), x = (int)(i % s.n[0]);
      w0[i] = unit_root(s.lo[0] + j, x, s.n[0]);
    } else if (i < e0 + e1) {
      const int64_t r = i - e0;
      const int j = (int)(r / s.n[1]), x = (int)(r % s.n[1]);
      w1[r] = unit_root(s.lo[1] + j, x, s.n[1]);
    } else if (i < e0 + e1 + e2) {
      const int64_t r = i - e0 - e1;
      const int j = (int)(r / s.ldw2), x = (int)(r % s.ldw2);
      w2[r] = x < s.n[2] ? unit_root(s.lo[2] + j, x, s.n[2]) : make_float2(0.f, 0.f);
    } else {
      const int64_t r = i - e0 - e1 - e2;
      const int x = (int)(r / s.ldj), j = (int)(r % s.ldj);
      float2 v = make_float2(0.f, 0.f);
      if (j < s.ext[2]) {
        v = unit_root(s.lo[2] + j, x, s.n[2]);
        v.y = -v.y;
      }
      w2t[r] = v;
    }
  }
}

// S = ft * OTF at the band voxels, written into the (zeroed) band box T0.
__device__ __forceinline__ void bb_scatter(const BBShape& s, const int32_t* __restrict__ band,
                                           int64_t m, const float2* __restrict__ ft,
                                           const float* __restrict__ otf,
                                           float2* __restrict__ t0, int* err) {
  const int32_t idx = band[m];
  if (idx < 0 || (int64_t)idx >= s.nvox) {
    set_error(err, DM_ERR_BAD_INDEX);
    return;
  }
  const int32_t n12 = s.n[1] * s.n[2];
  const int32_t k0 = idx / n12, rem = idx - k0 * n12;
  const int32_t k1 = rem / s.n[2], k2 = rem - k1 * s.n[2];
  const int32_t j0 = k0 - s.lo[0], j1 = k1 - s.lo[1], j2 = k2 - s.lo[2];
  if (j0 < 0 || j0 >= s.ext[0] || j1 < 0 || j1 >= s.ext[1] || j2 < 0 || j2 >= s.ext[2]) {
    set_error(err, DM_ERR_BAD_INDEX);
    return;
  }
  const float o = otf ? otf[idx] : 1.0f;
  const float2 f = ft[m];
  t0[((int64_t)j0 * s.ext[1] + j1) * s.ext[2] + j2] = make_float2(f.x * o, f.y * o);
}

__global__ void k_bb_scatter(BBShape s, const int32_t* __restrict__ band, int64_t nb,
                             const float2* __restrict__ ft, const float* __restrict__ otf,
                             float2* __restrict__ t0, int* err) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m < nb) bb_scatter(s, band, m, ft, otf, t0, err);
}

// ---------------------------------------------------------------------------
// Small batched complex GEMM with a root table on the left:
//   C[kp][b][m][n] = sum_{k in split kp} A(m, k) X[b][k][n]  (C strides scp, scb, scm, scn),
//   X = the sum (in order) of ``xparts`` arrays sxp elements apart,
//   kInv:  A(m, k) = W[k * ldw + m]        (inverse pass: m = position, k = band offset)
//   else:  A(m, k) = conj(W[m * ldw + k])  (forward pass: m = band offset, k = position)
// blockIdx.z = kp * batch + b; split kp covers k in [kp kc, (kp+1) kc) and writes its
// partial sums at C + kp * scp.  Tile 64 (m) x 32 (n), k in steps of 16 through
// shared memory with the next step's tiles loaded into registers while the current
// one is used; each thread owns 4 x 2 outputs.

struct GemmP {
  const float2* W;
  int ldw, M, N, K, batch, kc, xparts;
  const float2* X;
  int64_t sxb, sxk, sxp;
  float2* C;
  int64_t scb, scm, scn, scp;
};

// One (16 RM) x 32 output tile (bx, by) of split / batch entry bz; each thread
// owns RM x 2 outputs (RM = 4: 64-row tiles; RM = 2: 32-row tiles, for products
// with few rows).
template <bool kInv, int RM = 4>
__device__ __forceinline__ void bb_gemm_tile(const GemmP& p, int bx, int by, int bz) {
  constexpr int TM = 16 * RM;   // tile rows
  constexpr int RA = TM / 16;   // A elements per thread and k step
  const float2* __restrict__ W = p.W;
  const float2* __restrict__ X = p.X;
  const int ldw = p.ldw, M = p.M, N = p.N, K = p.K, batch = p.batch, kc = p.kc;
  const int xparts = p.xparts;
  const int64_t sxb = p.sxb, sxk = p.sxk, sxp = p.sxp;
  // rows padded by 16 bytes: the forward pass stores A with k across the lanes
  __shared__ __align__(16) float2 As[16][TM + 2];
  __shared__ __align__(16) float2 Bs[16][32];
  const int t = threadIdx.x;
  const int tm = t >> 4, tn = t & 15;
  const int m0 = by * TM, n0 = bx * 32;
  const int64_t b = bz % batch;
  const int kp = bz / batch;
  const int kb = kp * kc, ke = min(K, kb + kc);
  const float2* Xb = X + b * sxb;
  float2 ra[RA], rb[2];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int r = 0; r < RA; ++r) {
      const int e = t + kGemmThreads * r;
      const int m = kInv ? (e % TM) : (e >> 4);
      const int k = kInv ? (e / TM) : (e & 15);
      float2 v = make_float2(0.f, 0.f);
      if (m0 + m < M && k0 + k < ke) {
        if (kInv) {
          v = W[(int64_t)(k0 + k) * ldw + m0 + m];
        } else {
          v = W[(int64_t)(m0 + m) * ldw + k0 + k];
          v.y = -v.y;
        }
      }
      ra[r] = v;
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int e = t + kGemmThreads * r;
      const int n = e & 31, k = e >> 5;
      float2 v = make_float2(0.f, 0.f);
      if (n0 + n < N && k0 + k < ke) {
        const float2* px = Xb + (int64_t)(k0 + k) * sxk + n0 + n;
        v = px[0];
        for (int p = 1; p < xparts; ++p) {
          const float2 q = px[p * sxp];
          v.x += q.x;
          v.y += q.y;
        }
      }
      rb[r] = v;
    }
  };
  float2 acc[RM][2];
#pragma unroll
  for (int i = 0; i < RM; ++i) acc[i][0] = acc[i][1] = make_float2(0.f, 0.f);
  if (kb < ke) fetch(kb);
  for (int k0 = kb; k0 < ke; k0 += 16) {
#pragma unroll
    for (int r = 0; r < RA; ++r) {
      const int e = t + kGemmThreads * r;
      const int m = kInv ? (e % TM) : (e >> 4);
      const int k = kInv ? (e / TM) : (e & 15);
      As[k][m] = ra[r];
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int e = t + kGemmThreads * r;
      Bs[e >> 5][e & 31] = rb[r];
    }
    __syncthreads();
    if (k0 + 16 < ke) fetch(k0 + 16);
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      float2 a[RM];
#pragma unroll
      for (int q = 0; q < RM / 2; ++q) {
        const float4 v = *reinterpret_cast<const float4*>(&As[kk][tm * RM + 2 * q]);
        a[2 * q] = make_float2(v.x, v.y);
        a[2 * q + 1] = make_float2(v.z, v.w);
      }
      const float4 bb = *reinterpret_cast<const float4*>(&Bs[kk][tn * 2]);
      const float2 bv[2] = {make_float2(bb.x, bb.y), make_float2(bb.z, bb.w)};
#pragma unroll
      for (int i = 0; i < RM; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j] = cmac(acc[i][j], a[i], bv[j]);
    }
    __syncthreads();
  }
  float2* Cb = p.C + kp * p.scp + b * p.scb;
#pragma unroll
  for (int i = 0; i < RM; ++i) {
    const int m = m0 + tm * RM + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int n = n0 + tn * 2 + j;
      if (n < N) Cb[(int64_t)m * p.scm + (int64_t)n * p.scn] = acc[i][j];
    }
  }
}

template <bool kInv, int RM>
__global__ void __launch_bounds__(kGemmThreads) k_bb_gemm(GemmP p) {
  bb_gemm_tile<kInv, RM>(p, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------
// Reductions by the last CTA of a pass: every CTA stores its partial, the CTA
// that finishes last (counter in the header) combines all partials in a fixed
// order, so the result does not depend on which CTA that is.

__device__ __forceinline__ MMC mmc_empty() {
  return MMC{INFINITY, -INFINITY, INT32_MAX, INT32_MAX, 0, 0};
}

__device__ __forceinline__ MMC mmc_load(const MMC* p) {
  MMC q;
  q.mn = __ldcg(&p->mn);
  q.mx = __ldcg(&p->mx);
  q.imn = __ldcg(&p->imn);
  q.imx = __ldcg(&p->imx);
  q.cmn = __ldcg(&p->cmn);
  q.cmx = __ldcg(&p->cmx);
  return q;
}

// Merge of one MMC per thread over the block; the result is valid in thread 0.
__device__ MMC block_mmc(MMC r, MMC* sh) {
  for (int o = 16; o > 0; o >>= 1) mmc_merge(r, mmc_shfl(r, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = r;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mmc_merge(r, sh[w]);
  __syncthreads();
  return r;
}

// True in every thread of the CTA that finished last (after its partial is out).
__device__ bool last_cta(unsigned int* counter, unsigned int total, int* flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int prev = atomicAdd(counter, 1u);
    *flag = prev == total - 1u;
  }
  __syncthreads();
  const bool last = *flag != 0;
  if (last) __threadfence();
  return last;
}

// ---------------------------------------------------------------------------
// z pass: persistent CTAs, each with one column block of 32*C positions x2
// (blockIdx.y) and the line tiles blockIdx.x, blockIdx.x + gridDim.x, ... of 32
// lines (x0, x1) each:
//   z[line][x2] = 1/N sum_j T2[line][j] W2[j][x2];  |z|, min / max.
// The W2 column block is staged once by bulk copies; the T2 rows of a tile arrive
// by bulk copy into one of two buffers while the previous tile is computed.
// Thread (warp w, lane l): lines 4w..4w+3, positions l + 32c.  The last CTA
// writes the min / max (first index, tie count) to the header.

__device__ __forceinline__ uint32_t zl_tile_bytes(const BBShape& s, int64_t tile) {
  const int64_t nl = min((int64_t)kLines, s.nlines - tile * kLines);
  return (uint32_t)((nl * s.ext[2] * (int64_t)sizeof(float2) + 15) & ~(int64_t)15);
}

// CTA (bx, by) of G x (column blocks) for one box.
template <int C>
__device__ __forceinline__ void bb_zlines(const BBShape& s, const float2* __restrict__ t2,
                                          const float2* __restrict__ w2, float inv_n,
                                          float2* __restrict__ z, float* __restrict__ image,
                                          MMC* __restrict__ part, BBHdr* hdr, int bx, int by,
                                          int G, int ncb) {
  extern __shared__ __align__(16) float2 sm[];
  __shared__ __align__(8) uint64_t bar[3];  // W2 block, T2 buffers 0 / 1
  __shared__ MMC shm[kLineThreads / 32];
  __shared__ int last;
  const int ext = s.ext[2], n2 = s.n[2];
  constexpr int Wc = 32 * C;
  float2* ws = sm;                        // [ext][Wc]
  float2* xs0 = sm + ext * Wc;            // [2][kLines][ext]
  const int64_t ntiles = (s.nlines + kLines - 1) / kLines;
  const int col0 = by * Wc;
  if (threadIdx.x == 0) {
    for (int b = 0; b < 3; ++b) mbar_init(&bar[b], 1);
    fence_mbar_init();
  }
  __syncthreads();
  // copies issued into each barrier and copies waited for (thread 0 drains the
  // difference if a wait gives up, before the CTA leaves)
  int iss_w = 0, iss_0 = 0, iss_1 = 0, got_w = 0, got_0 = 0, got_1 = 0;
  if (threadIdx.x == 0) {
    const uint32_t wb = (uint32_t)(Wc * sizeof(float2));
    mbar_expect_tx(&bar[0], (uint32_t)ext * wb);
    for (int j = 0; j < ext; ++j)
      bulk_g2s(ws + j * Wc, w2 + (int64_t)j * s.ldw2 + col0, wb, &bar[0]);
    iss_w = 1;
    for (int b = 0; b < 2; ++b) {
      const int64_t tile = bx + (int64_t)b * G;
      if (tile >= ntiles) break;
      const uint32_t xb = zl_tile_bytes(s, tile);
      mbar_expect_tx(&bar[1 + b], xb);
      bulk_g2s(xs0 + b * kLines * ext, t2 + tile * kLines * ext, xb, &bar[1 + b]);
      if (b == 0) iss_0 = 1; else iss_1 = 1;
    }
  }
  bool ok = __syncthreads_and(mbar_wait_sleep_bounded(&bar[0], 0, &hdr->err));
  got_w = ok ? 1 : 0;
  const int ty = threadIdx.x >> 5, tx = threadIdx.x & 31;
  MMC r = mmc_empty();
  int it = 0;
  for (int64_t tile = bx; ok && tile < ntiles; tile += G, ++it) {
    const int buf = it & 1;
    ok = __syncthreads_and(mbar_wait_sleep_bounded(&bar[1 + buf], (it >> 1) & 1, &hdr->err));
    if (!ok) break;
    if (buf == 0) ++got_0; else ++got_1;
    const float2* xs = xs0 + buf * kLines * ext;
    float2 acc[4][C];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int c = 0; c < C; ++c) acc[i][c] = make_float2(0.f, 0.f);
    for (int j = 0; j < ext; ++j) {
      float2 xv[4], wv[C];
#pragma unroll
      for (int i = 0; i < 4; ++i) xv[i] = xs[(ty * 4 + i) * ext + j];
#pragma unroll
      for (int c = 0; c < C; ++c) wv[c] = ws[j * Wc + tx + 32 * c];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int c = 0; c < C; ++c) acc[i][c] = cmac(acc[i][c], xv[i], wv[c]);
    }
    __syncthreads();  // every read of this buffer is done: refill it
    if (threadIdx.x == 0 && tile + 2 * (int64_t)G < ntiles) {
      fence_proxy_async();
      const uint32_t xb = zl_tile_bytes(s, tile + 2 * (int64_t)G);
      mbar_expect_tx(&bar[1 + buf], xb);
      bulk_g2s(xs0 + buf * kLines * ext, t2 + (tile + 2 * (int64_t)G) * kLines * ext, xb,
               &bar[1 + buf]);
      if (buf == 0) ++iss_0; else ++iss_1;
    }
    const int64_t line0 = tile * kLines;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int64_t line = line0 + ty * 4 + i;
      if (line >= s.nlines) continue;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int x = col0 + tx + 32 * c;
        if (x >= n2) continue;
        const float2 v = make_float2(acc[i][c].x * inv_n, acc[i][c].y * inv_n);
        const int32_t idx = (int32_t)(line * n2 + x);
        z[idx] = v;
        const float a = cabs2(v);
        if (image) image[idx] = a;
        mmc_add(r, a, idx);
      }
    }
  }
  if (!ok && threadIdx.x == 0) {  // a wait gave up: let the copies in flight land first
    if (iss_w > got_w) mbar_wait_sleep_bounded(&bar[0], 0, &hdr->err);
    if (iss_0 > got_0) mbar_wait_sleep_bounded(&bar[1], (iss_0 - 1) & 1, &hdr->err);
    if (iss_1 > got_1) mbar_wait_sleep_bounded(&bar[2], (iss_1 - 1) & 1, &hdr->err);
  }
  r = block_mmc(r, shm);
  const unsigned int total = (unsigned int)G * ncb;
  if (threadIdx.x == 0) part[(int64_t)by * G + bx] = r;
  if (!last_cta(&hdr->done[0], total, &last)) return;
  MMC q = mmc_empty();
  for (unsigned int b = threadIdx.x; b < total; b += blockDim.x) mmc_merge(q, mmc_load(part + b));
  q = block_mmc(q, shm);
  if (threadIdx.x == 0) {
    hdr->mn = q.mn;
    hdr->mx = q.mx;
    hdr->imn = q.imn;
    hdr->imx = q.imx;
    hdr->cmn = q.cmn;
    hdr->cmx = q.cmx;
    hdr->done[0] = 0u;  // every CTA has counted: ready for the next call
  }
}

template <int C>
__global__ void __launch_bounds__(kLineThreads)
    k_bb_zlines(BBShape s, const float2* __restrict__ t2, const float2* __restrict__ w2,
                float inv_n, float2* __restrict__ z, float* __restrict__ image,
                MMC* __restrict__ part, BBHdr* hdr) {
  bb_zlines<C>(s, t2, w2, inv_n, z, image, part, hdr, blockIdx.x, blockIdx.y, gridDim.x,
               gridDim.y);
}

// ---------------------------------------------------------------------------
// Gradient pass: per voxel of 32 lines the normalised image, the loss term and
// g = dL/dz without the min / max terms (the same float arithmetic as
// dm_image_loss), staged transposed in shared memory; then
//   Q2[line][j] = sum_x2 g[line][x2] conj(W2[j][x2])
// with warp w summing x2 in [w n2/8, (w+1) n2/8) for 4 lines x 2JC band offsets
// per thread, and the eight warp partials added in warp order.  The conjugate
// table arrives by a bulk copy while the voxels are processed.  Voxels go to the
// warps in tiles of 4 lines x 8 positions (coalesced 64-byte row pieces), read
// kAhead tiles ahead.  The transposed tile gT[x2][line] swaps groups of 4 lines
// by x2 mod 8 and the partial sums swap 16-byte units by line, so neither the
// stores nor the reads of either meet bank conflicts.  The last CTA forms the
// loss and the min / max gradient per tied voxel.

constexpr int kAhead = 8;  // voxel tiles per warp loaded before use

// Band offsets j are contracted in chunks of at most 32 (8 JC per chunk); an
// extent above 32 takes two chunks, the partial sums of a chunk then have their
// own area instead of reusing the voxel tile's.
__host__ __device__ inline int grad_chunk(int ldj) { return ldj <= 32 ? ldj : 32; }
__host__ __device__ inline int red_units(int ldj) {  // 16-byte units per partial-sum row
  const int u = grad_chunk(ldj) / 2;
  return u <= 8 ? 8 : 16;
}

size_t gradlines_smem(int n2, int ldj) {
  const size_t gz = (size_t)n2 * kLines * sizeof(float2);
  const size_t rd = (size_t)8 * kLines * red_units(ldj) * 16;
  const size_t tile = ldj <= 32 ? std::max(gz, rd) : gz + rd;
  return (size_t)n2 * ldj * sizeof(float2) + tile;
}

// CTA bx of G for one box.
template <int JC>
__device__ __forceinline__ void bb_gradlines(const BBShape& s, const float2* __restrict__ z,
                                             const float* __restrict__ target, int kind,
                                             float contrast, BBHdr* hdr,
                                             const float2* __restrict__ w2t,
                                             float2* __restrict__ q2, LP* __restrict__ part,
                                             float* __restrict__ loss, int bx, int G) {
  extern __shared__ __align__(16) float2 sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ double shl[3][kLineThreads / 32];
  __shared__ LP shp[kLineThreads];
  __shared__ int last;
  const int n2 = s.n[2], ext = s.ext[2], ldj = s.ldj;
  float2* wt = sm;                 // [n2][ldj], staged once
  float2* gzt = sm + n2 * ldj;     // [n2][kLines], line groups swizzled by x2 mod 8
  // [8][kLines][RU] 16-byte units: after the contraction over the voxel tile, or
  // after it when there are two chunks
  float4* red = reinterpret_cast<float4*>(ldj <= 32 ? gzt : gzt + n2 * kLines);
  const int RU = red_units(ldj);
  const int64_t ntiles = (s.nlines + kLines - 1) / kLines;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t bytes = (uint32_t)((size_t)n2 * ldj * sizeof(float2));
    mbar_expect_tx(&bar, bytes);
    bulk_g2s(wt, w2t, bytes, &bar);
  }
  const float mn = hdr->mn, mx = hdr->mx;
  const float rng = mx - mn;
  const float inv = 1.0f / (rng * (1.0f + contrast));
  const float inv_rng = 1.0f / rng, inv_1c = 1.0f / (1.0f + contrast);
  const float nseg_inv = 1.0f / (float)s.nvox;
  double L = 0.0, dmn = 0.0, dmx = 0.0;
  // phase 1 mapping: warp w, lines 4w..4w+3; lane = 8 li + xi: line 4w+li, position
  // 8k+xi of position tile k.  GEMM mapping: lane = lg + 8 jg.
  const int li = lane >> 3, xi = lane & 7;
  const int l = 4 * w + li;
  const int col = (l ^ (xi << 2));  // gT column of this lane's line (x2 mod 8 == xi)
  const int ntile = (n2 + 7) / 8;
  const int lg = lane & 7, jg = lane >> 3;
  bool ok = true, staged = false;
  for (int64_t tile = bx; tile < ntiles; tile += G) {
    const int64_t line0 = tile * kLines;
    const int64_t line = line0 + l;
    const bool live_line = line < s.nlines;
    for (int k0 = 0; k0 < ntile; k0 += kAhead) {
      float2 zv[kAhead];
      float tv[kAhead];
#pragma unroll
      for (int u = 0; u < kAhead; ++u) {
        const int x = 8 * (k0 + u) + xi;
        const bool live = live_line && x < n2;
        const int64_t i = line * n2 + x;
        zv[u] = live ? z[i] : make_float2(0.f, 0.f);
        tv[u] = (live && kind != 0) ? target[i] : 0.f;
      }
#pragma unroll
      for (int u = 0; u < kAhead; ++u) {
        const int x = 8 * (k0 + u) + xi;
        if (x >= n2) continue;
        float2 g = make_float2(0.f, 0.f);
        if (live_line) {
          const float2 zi = zv[u];
          const float a = cabs2(zi);
          // reciprocals of the per-image constants instead of divisions (ulp-level
          // differences from dm_image_loss)
          const float uu = (a - mn) * inv_rng;
          const float nv = contrast == 0.0f ? uu : (uu + contrast) * inv_1c;
          float gn;
          if (kind == 0) {
            L += nv;
            gn = 1.0f;
          } else if (kind == 1) {
            const float dlt = nv - tv[u];
            L += (double)dlt * dlt;
            gn = 2.0f * dlt * nseg_inv;
          } else {
            gn = tv[u];  // kind 2: dL/d|z| given, no normalisation
          }
          if (kind != 2) {
            dmn += (double)gn * (-(1.0 - (double)uu));
            dmx += (double)gn * (-(double)uu);
          }
          const float gg = kind == 2 ? gn : gn * inv;
          const float sc = a > 0.f ? __fdividef(gg, a) : 0.f;
          g = make_float2(sc * zi.x, sc * zi.y);
        }
        gzt[x * kLines + col] = g;
      }
    }
    if (!staged) {
      ok = __syncthreads_and(mbar_wait_sleep_bounded(&bar, 0, &hdr->err));
      staged = true;
      if (!ok) break;
    }
    __syncthreads();
    for (int jc0 = 0; jc0 < ldj; jc0 += 8 * JC) {
      const int jn = min(JC, (ldj - jc0) >> 3);  // 8-offset groups in this chunk
      float2 acc[4][JC][2];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int c = 0; c < JC; ++c) acc[i][c][0] = acc[i][c][1] = make_float2(0.f, 0.f);
      const int xb = w * n2 / 8, xe = (w + 1) * n2 / 8;
      for (int x = xb; x < xe; ++x) {
        const int grp = lg ^ (x & 7);
        const float2* row = gzt + x * kLines + 4 * grp;  // lines 4lg..4lg+3
        // groups 4..7 read their second half first: the eight lanes of a quarter
        // warp then cover all 32 banks in each of the two 16-byte loads
        const int h = (grp >> 2) & 1;
        const float4 ga = *reinterpret_cast<const float4*>(row + 2 * h);
        const float4 gb = *reinterpret_cast<const float4*>(row + 2 - 2 * h);
        const float4 g01 = h ? gb : ga, g23 = h ? ga : gb;
        const float2 gv[4] = {make_float2(g01.x, g01.y), make_float2(g01.z, g01.w),
                              make_float2(g23.x, g23.y), make_float2(g23.z, g23.w)};
#pragma unroll
        for (int c = 0; c < JC; ++c) {
          if (c >= jn) break;
          const float4 wv =
              *reinterpret_cast<const float4*>(&wt[x * ldj + jc0 + c * 8 + jg * 2]);
          const float2 w0 = make_float2(wv.x, wv.y), w1 = make_float2(wv.z, wv.w);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            acc[i][c][0] = cmac(acc[i][c][0], gv[i], w0);
            acc[i][c][1] = cmac(acc[i][c][1], gv[i], w1);
          }
        }
      }
      __syncthreads();
      // partial sums: row (warp, line), 16-byte unit (c*4 + jg) ^ (line >> 2)
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int ln = lg * 4 + i;
#pragma unroll
        for (int c = 0; c < JC; ++c)
          if (c < jn)
            red[(w * kLines + ln) * RU + ((c * 4 + jg) ^ lg)] =
                make_float4(acc[i][c][0].x, acc[i][c][0].y, acc[i][c][1].x, acc[i][c][1].y);
      }
      __syncthreads();
      const int je = min(8 * jn, ext - jc0);  // band offsets of this chunk
      for (int e = threadIdx.x; e < kLines * je; e += kLineThreads) {
        const int ln = e / je, j = e - ln * je;
        const int64_t lq = line0 + ln;
        if (lq >= s.nlines) continue;
        const int unit = (j >> 1) ^ (ln >> 2);
        const float* base = reinterpret_cast<const float*>(red) + 4 * unit + 2 * (j & 1);
        float2 v = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const float* p = base + 4 * (k * kLines + ln) * RU;
          v.x += p[0];
          v.y += p[1];
        }
        q2[lq * ext + jc0 + j] = v;
      }
      __syncthreads();  // red (and, with one chunk, the voxel tile) is written again
    }
  }
  if (!staged && threadIdx.x == 0) mbar_wait_sleep_bounded(&bar, 0, &hdr->err);
  if (!ok && threadIdx.x == 0) mbar_wait_sleep_bounded(&bar, 0, &hdr->err);
  // loss partials (fixed order)
  double v[3] = {L, dmn, dmx};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double x = v[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) shl[k][w] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    LP r{0.0, 0.0, 0.0};
    for (int k = 0; k < kLineThreads / 32; ++k) {
      r.loss += shl[0][k];
      r.dmn += shl[1][k];
      r.dmx += shl[2][k];
    }
    part[bx] = r;
  }
  if (!last_cta(&hdr->done[1], (unsigned int)G, &last)) return;
  LP r{0.0, 0.0, 0.0};
  for (unsigned int k = threadIdx.x; k < (unsigned int)G; k += blockDim.x) {
    r.loss += __ldcg(&part[k].loss);
    r.dmn += __ldcg(&part[k].dmn);
    r.dmx += __ldcg(&part[k].dmx);
  }
  shp[threadIdx.x] = r;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      shp[threadIdx.x].loss += shp[threadIdx.x + o].loss;
      shp[threadIdx.x].dmn += shp[threadIdx.x + o].dmn;
      shp[threadIdx.x].dmx += shp[threadIdx.x + o].dmx;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const LP q = shp[0];
    const double drng = (double)hdr->mx - (double)hdr->mn;
    const double dinv = 1.0 / (drng * (1.0 + contrast));
    const double f0 = kind == 0 ? q.loss : q.loss / (double)s.nvox;
    const double f1 = q.dmn * dinv, f2 = q.dmx * dinv;
    hdr->fin[0] = f0;
    hdr->fin[1] = f1;
    hdr->fin[2] = f2;
    hdr->add_mn = hdr->cmn > 0 ? (float)(f1 / (double)hdr->cmn) : 0.f;
    hdr->add_mx = hdr->cmx > 0 ? (float)(f2 / (double)hdr->cmx) : 0.f;
    hdr->ties_full = (kind != 2 && (hdr->cmn >= 2 || hdr->cmx >= 2)) ? 1 : 0;
    if (loss) loss[0] = (float)f0;
    hdr->done[1] = 0u;  // every CTA has counted: ready for the next call
  }
}

template <int JC>
__global__ void __launch_bounds__(kLineThreads)
    k_bb_gradlines(BBShape s, const float2* __restrict__ z, const float* __restrict__ target,
                   int kind, float contrast, BBHdr* hdr, const float2* __restrict__ w2t,
                   float2* __restrict__ q2, LP* __restrict__ part, float* __restrict__ loss) {
  bb_gradlines<JC>(s, z, target, kind, contrast, hdr, w2t, q2, part, loss, blockIdx.x,
                   gridDim.x);
}

// Several voxels at the min (max): add their share of the min (max) gradient to
// the line contractions, one thread per line in x2 order.  Returns at once in the
// usual case of a single voxel (added in the gather instead).
__device__ __forceinline__ void bb_ties(const BBShape& s, const float2* __restrict__ z,
                                        const BBHdr* __restrict__ hdr,
                                        const float2* __restrict__ w2t, float2* __restrict__ q2,
                                        int64_t line) {
  if (!hdr->ties_full) return;
  if (line >= s.nlines) return;
  const bool t0 = hdr->cmn >= 2, t1 = hdr->cmx >= 2;
  const float mn = hdr->mn, mx = hdr->mx, a0 = hdr->add_mn, a1 = hdr->add_mx;
  const int n2 = s.n[2], ext = s.ext[2];
  for (int x = 0; x < n2; ++x) {
    const float2 zi = z[line * n2 + x];
    const float a = cabs2(zi);
    const bool h0 = t0 && a == mn, h1 = t1 && a == mx;
    if (!(h0 || h1) || !(a > 0.f)) continue;
    for (int k = 0; k < 2; ++k) {
      if (!(k == 0 ? h0 : h1)) continue;
      const float sc = (k == 0 ? a0 : a1) / a;
      const float2 v = make_float2(sc * zi.x, sc * zi.y);
      for (int j = 0; j < ext; ++j)
        q2[line * ext + j] = cmac(q2[line * ext + j], v, w2t[(int64_t)x * s.ldj + j]);
    }
  }
}

__global__ void k_bb_ties(BBShape s, const float2* __restrict__ z, const BBHdr* __restrict__ hdr,
                          const float2* __restrict__ w2t, float2* __restrict__ q2) {
  bb_ties(s, z, hdr, w2t, q2, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// Axis-0 forward contraction into the band box, one CTA per column (j1, j2):
//   G0[j0][j1 j2] = sum_x0 conj(W0[j0][x0]) Q1[j1 j2][x0]
// with Q1 the sum (in order) of its K-split partials, staged in shared memory
// from its column-major layout; eight lanes per output, fixed shuffle tree.
constexpr int kColThreads = 128;

__device__ __forceinline__ void bb_columns(const BBShape& s, const float2* __restrict__ q1t,
                                           const float2* __restrict__ w0,
                                           float2* __restrict__ g0, int64_t c) {
  extern __shared__ __align__(16) float2 colv[];  // [n0]; c = j1 * ext2 + j2
  const int64_t ncol = (int64_t)s.ext[1] * s.ext[2];
  const int n0 = s.n[0];
  for (int x0 = threadIdx.x; x0 < n0; x0 += kColThreads) {
    const float2* p = q1t + c * n0 + x0;
    float2 q = p[0];
    for (int kp = 1; kp < s.q1split; ++kp) {
      const float2 r = p[kp * ncol * n0];
      q.x += r.x;
      q.y += r.y;
    }
    colv[x0] = q;
  }
  __syncthreads();
  const int sub = threadIdx.x & 7, grp = threadIdx.x >> 3;
  const int rounds = (s.ext[0] + kColThreads / 8 - 1) / (kColThreads / 8);
  for (int it = 0; it < rounds; ++it) {  // the same rounds for every lane (shuffles)
    const int j0 = grp + it * (kColThreads / 8);
    float2 g = make_float2(0.f, 0.f);
    if (j0 < s.ext[0]) {
      const float2* wr = w0 + (int64_t)j0 * n0;
#pragma unroll 5
      for (int x0 = sub; x0 < n0; x0 += 8) {
        float2 w = wr[x0];
        w.y = -w.y;
        g = cmac(g, colv[x0], w);
      }
    }
    for (int o = 4; o > 0; o >>= 1) {
      g.x += __shfl_down_sync(0xffffffffu, g.x, o, 8);
      g.y += __shfl_down_sync(0xffffffffu, g.y, o, 8);
    }
    if (sub == 0 && j0 < s.ext[0]) g0[(int64_t)j0 * ncol + c] = g;
  }
}

__global__ void __launch_bounds__(kColThreads)
    k_bb_columns(BBShape s, const float2* __restrict__ q1t, const float2* __restrict__ w0,
                 float2* __restrict__ g0) {
  bb_columns(s, q1t, w0, g0, blockIdx.x);
}

// G at the band voxels: G0 plus the min / max gradient of a single extreme voxel.
__device__ __forceinline__ float2 bb_gather(const BBShape& s, const int32_t* __restrict__ band,
                                           int64_t m, const float2* __restrict__ g0,
                                           const float2* __restrict__ w0,
                                           const float2* __restrict__ w1,
                                           const float2* __restrict__ w2,
                                           const float2* __restrict__ z,
                                           const BBHdr* __restrict__ hdr) {
  int32_t idx = band[m];
  if (idx < 0 || (int64_t)idx >= s.nvox) idx = 0;  // reported by the scatter
  const int32_t n12 = s.n[1] * s.n[2];
  const int32_t k0 = idx / n12, rem = idx - k0 * n12;
  const int32_t k1 = rem / s.n[2], k2 = rem - k1 * s.n[2];
  const int32_t j0 = min(max(k0 - s.lo[0], 0), s.ext[0] - 1);
  const int32_t j1 = min(max(k1 - s.lo[1], 0), s.ext[1] - 1);
  const int32_t j2 = min(max(k2 - s.lo[2], 0), s.ext[2] - 1);
  float2 g = g0[((int64_t)j0 * s.ext[1] + j1) * s.ext[2] + j2];
  if (!hdr->ties_full) {
    for (int k = 0; k < 2; ++k) {
      const int64_t c = k == 0 ? hdr->cmn : hdr->cmx;
      if (c != 1) continue;
      const int64_t i = k == 0 ? hdr->imn : hdr->imx;
      const float2 zi = z[i];
      const float a = cabs2(zi);
      const float sc = a > 0.f ? (k == 0 ? hdr->add_mn : hdr->add_mx) / a : 0.f;
      const float2 v = make_float2(sc * zi.x, sc * zi.y);
      const int64_t nn12 = (int64_t)s.n[1] * s.n[2];
      const int x0 = (int)(i / nn12), x1 = (int)((i / s.n[2]) % s.n[1]), x2 = (int)(i % s.n[2]);
      float2 e = cmulf(cmulf(w0[(int64_t)j0 * s.n[0] + x0], w1[(int64_t)j1 * s.n[1] + x1]),
                       w2[(int64_t)j2 * s.ldw2 + x2]);
      e.y = -e.y;
      g = cmac(g, v, e);
    }
  }
  return g;
}

__global__ void k_bb_gather(BBShape s, const int32_t* __restrict__ band, int64_t nb,
                            const float2* __restrict__ g0, const float2* __restrict__ w0,
                            const float2* __restrict__ w1, const float2* __restrict__ w2,
                            const float2* __restrict__ z, const BBHdr* __restrict__ hdr,
                            float2* __restrict__ grad_list) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m < nb) grad_list[m] = bb_gather(s, band, m, g0, w0, w1, w2, z, hdr);
}

// Band bounding box: per axis the smallest and largest index of the band
// (integer atomics: order-independent).
__global__ void k_bb_bounds(const int32_t* __restrict__ band, int64_t nb, int32_t n1, int32_t n2,
                            int32_t* __restrict__ out) {
  int32_t lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {-1, -1, -1};
  for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < nb;
       m += (int64_t)gridDim.x * blockDim.x) {
    const int32_t idx = band[m];
    if (idx < 0) continue;
    const int32_t n12 = n1 * n2;
    const int32_t k[3] = {idx / n12, (idx / n2) % n1, idx % n2};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      lo[d] = min(lo[d], k[d]);
      hi[d] = max(hi[d], k[d]);
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = min(lo[d], __shfl_down_sync(0xffffffffu, lo[d], o));
      hi[d] = max(hi[d], __shfl_down_sync(0xffffffffu, hi[d], o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&out[d], lo[d]);
      atomicMax(&out[3 + d], hi[d]);
    }
  }
}

__global__ void k_bb_bounds_init(int32_t* out) {
  if (threadIdx.x < 3) {
    out[threadIdx.x] = INT32_MAX;
    out[3 + threadIdx.x] = -1;
  }
}

// ---------------------------------------------------------------------------
// Workspace layout.

size_t up256(size_t x) { return (x + 255) / 256 * 256; }

struct BBWs {
  BBHdr* hdr;
  float2 *w0, *w1, *w2, *w2t;
  float2 *t0, *t1, *t2;  // band box, after axis 0, after axis 1 (Q2 reuses t2)
  float2* q1p;           // K-split partials of the axis-1 forward contraction
  float2* g0;            // axis-0 forward contraction over the band box
  float2* z;
  MMC* mm;
  LP* lp;
};

int z_col_chunk(int n2) { return std::min(8, (n2 + 31) / 32); }

size_t bb_layout(const BBShape& s, char* base, BBWs* w) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> char* {
    char* p = base ? base + off : nullptr;
    off += up256(std::max<size_t>(bytes, 1) + 16);  // 16 bytes of slack: rounded bulk copies
    return p;
  };
  const size_t c8 = sizeof(float2);
  const int64_t e0 = s.ext[0], e1 = s.ext[1], e2 = s.ext[2];
  const int64_t nlb = (s.nlines + kLines - 1) / kLines;
  const int64_t cb = s.ldw2 / (32 * s.zc);
  BBWs r;
  r.hdr = (BBHdr*)take(sizeof(BBHdr));
  r.w0 = (float2*)take(c8 * e0 * s.n[0]);
  r.w1 = (float2*)take(c8 * e1 * s.n[1]);
  r.w2 = (float2*)take(c8 * e2 * s.ldw2);
  r.w2t = (float2*)take(c8 * (size_t)s.n[2] * s.ldj);
  r.t0 = (float2*)take(c8 * e0 * e1 * e2);
  r.t1 = (float2*)take(c8 * (size_t)s.n[0] * e1 * e2);
  r.t2 = (float2*)take(c8 * (size_t)s.nlines * e2);
  r.q1p = (float2*)take(c8 * (size_t)s.q1split * s.n[0] * e1 * e2);
  r.g0 = (float2*)take(c8 * e0 * e1 * e2);
  r.z = (float2*)take(c8 * (size_t)s.nvox);
  r.mm = (MMC*)take(sizeof(MMC) * (size_t)(nlb * cb));
  r.lp = (LP*)take(sizeof(LP) * (size_t)nlb);
  if (w) *w = r;
  return off;
}

// K split of a forward contraction over n positions: (chunk, splits), chunk a
// multiple of 16.
void ksplit(int n, int& chunk, int& splits) {
  const int want = std::max(1, std::min(8, n / 48));
  chunk = ((n + want - 1) / want + 15) / 16 * 16;
  splits = (n + chunk - 1) / chunk;
}

bool make_shape(const int32_t n[3], const int32_t lo[3], const int32_t ext[3], BBShape& s) {
  for (int d = 0; d < 3; ++d) {
    if (n[d] <= 0 || ext[d] <= 0 || lo[d] < 0 || (int64_t)lo[d] + ext[d] > n[d]) return false;
    s.n[d] = n[d];
    s.lo[d] = lo[d];
    s.ext[d] = ext[d];
  }
  s.ldj = (ext[2] + 7) / 8 * 8;
  s.zc = z_col_chunk(n[2]);
  s.ldw2 = (n[2] + 32 * s.zc - 1) / (32 * s.zc) * (32 * s.zc);
  ksplit(n[1], s.q1chunk, s.q1split);
  s.nlines = (int64_t)n[0] * n[1];
  s.nvox = s.nlines * n[2];
  return s.nvox <= (int64_t)INT32_MAX && (int64_t)n[0] * s.q1split <= 65535 && n[0] <= 4096 &&
         s.nlines / kLines < (int64_t)INT32_MAX;
}

GemmP gemm_p(const float2* W, int ldw, int M, int N, int K, int kc, const float2* X,
             int64_t sxb, int64_t sxk, int xparts, int64_t sxp, float2* C, int64_t scb,
             int64_t scm, int64_t scn, int64_t scp, int batch) {
  GemmP p;
  p.W = W; p.ldw = ldw; p.M = M; p.N = N; p.K = K; p.batch = batch; p.kc = kc;
  p.xparts = xparts; p.X = X; p.sxb = sxb; p.sxk = sxk; p.sxp = sxp;
  p.C = C; p.scb = scb; p.scm = scm; p.scn = scn; p.scp = scp;
  return p;
}

// grid of one product: N tiles, M tiles (of 16 rm rows), batch x K splits
dim3 gemm_grid(const GemmP& p, int rm = 4) {
  const int splits = (p.K + p.kc - 1) / p.kc;
  return dim3((p.N + 31) / 32, (p.M + 16 * rm - 1) / (16 * rm), p.batch * splits);
}

// The axis-1 forward contraction has few rows (band offsets j1): 32-row tiles.
template <bool kInv>
void gemm(const float2* W, int ldw, int M, int N, int K, int kc, const float2* X, int64_t sxb,
          int64_t sxk, int xparts, int64_t sxp, float2* C, int64_t scb, int64_t scm,
          int64_t scn, int64_t scp, int batch, cudaStream_t st) {
  const GemmP p = gemm_p(W, ldw, M, N, K, kc, X, sxb, sxk, xparts, sxp, C, scb, scm, scn, scp,
                         batch);
  if (kInv)
    k_bb_gemm<kInv, 4><<<gemm_grid(p, 4), kGemmThreads, 0, st>>>(p);
  else
    k_bb_gemm<kInv, 2><<<gemm_grid(p, 2), kGemmThreads, 0, st>>>(p);
}


// Raises a kernel's dynamic shared-memory limit to kSmemLimit, once per device
// (a host-side attribute, set on the first call, before any stream capture).
template <typename Kern>
cudaError_t smem_limit_once(Kern k, std::atomic<bool>* done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < 64 && done[dev].load()) return cudaSuccess;
  e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimit);
  if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev].store(true);
  return e;
}

// Persistent CTAs of the line passes: two per SM, never more than the tiles.
int line_ctas(int64_t tiles) { return (int)std::max<int64_t>(1, std::min<int64_t>(tiles, 2 * num_sms())); }

size_t zlines_smem(const BBShape& s) {
  return sizeof(float2) * ((size_t)s.ext[2] * 32 * s.zc + 2 * (size_t)kLines * s.ext[2]);
}

template <int C>
cudaError_t zlines(const BBShape& s, const BBWs& w, float inv_n, float* image, cudaStream_t st) {
  const size_t smem = zlines_smem(s);
  auto k = k_bb_zlines<C>;
  static std::atomic<bool> done[64];
  cudaError_t e = smem_limit_once(k, done);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)line_ctas((s.nlines + kLines - 1) / kLines), s.ldw2 / (32 * C));
  k<<<grid, kLineThreads, smem, st>>>(s, w.t2, w.w2, inv_n, w.z, image, w.mm, w.hdr);
  return cudaGetLastError();
}

template <int JC>
cudaError_t gradlines(const BBShape& s, const BBWs& w, int kind, const float* target,
                      float contrast, float* loss, cudaStream_t st) {
  const size_t smem = gradlines_smem(s.n[2], s.ldj);
  auto k = k_bb_gradlines<JC>;
  static std::atomic<bool> done[64];
  cudaError_t e = smem_limit_once(k, done);
  if (e != cudaSuccess) return e;
  const unsigned nb = (unsigned)line_ctas((s.nlines + kLines - 1) / kLines);
  k<<<nb, kLineThreads, smem, st>>>(s, w.z, target, kind, contrast, w.hdr, w.w2t, w.t2, w.lp,
                                    loss);
  return cudaGetLastError();
}


// ---------------------------------------------------------------------------
// Many boxes per launch (the cells of a batch).  Each stage is one launch over
// all cells (the z and gradient passes: one per distinct template parameter),
// blockIdx.z (or the flat element index) selecting the cell; CTAs past a cell's
// own grid return at once.  Per cell the work and every sum are those of the
// single-box call.

struct BBCell {
  BBShape s;
  BBWs w;
  int64_t band_off, nband, grid_off;
  int32_t zctas, zcb, gctas, e12;
  float inv_n, gscale;
};

// Largest c in [0, n) with pref[c] <= x (pref ascending, pref[0] = 0).
template <typename T>
__device__ __forceinline__ int find_cell(const T* __restrict__ pref, int n, T x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pref[mid] <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void k_bbb_scatter(const BBCell* __restrict__ cells, const int64_t* __restrict__ bpref,
                              int ncells, int64_t total, const int32_t* __restrict__ band,
                              const float2* __restrict__ ft, const float* __restrict__ otf) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= total) return;
  const int c = find_cell(bpref, ncells, m);
  const BBCell& cc = cells[c];
  bb_scatter(cc.s, band + cc.band_off, m - cc.band_off, ft + cc.band_off,
             otf ? otf + cc.grid_off : nullptr, cc.w.t0, &cc.w.hdr->err);
}

template <bool kInv>
__global__ void __launch_bounds__(kGemmThreads)
    k_bbb_gemm(const GemmP* __restrict__ ps, const int32_t* __restrict__ zp, int ncells) {
  constexpr int RM = kInv ? 4 : 2;
  const int c = find_cell(zp, ncells, (int32_t)blockIdx.z);
  const GemmP p = ps[c];
  if ((int)blockIdx.x * 32 >= p.N || (int)blockIdx.y * 16 * RM >= p.M) return;
  bb_gemm_tile<kInv, RM>(p, blockIdx.x, blockIdx.y, (int)blockIdx.z - zp[c]);
}

template <int C>
__global__ void __launch_bounds__(kLineThreads)
    k_bbb_zlines(const BBCell* __restrict__ cells, const int32_t* __restrict__ order,
                 float* __restrict__ image) {
  const BBCell& cc = cells[order[blockIdx.z]];
  if ((int)blockIdx.x >= cc.zctas || (int)blockIdx.y >= cc.zcb) return;
  bb_zlines<C>(cc.s, cc.w.t2, cc.w.w2, cc.inv_n, cc.w.z, image ? image + cc.grid_off : nullptr,
               cc.w.mm, cc.w.hdr, blockIdx.x, blockIdx.y, cc.zctas, cc.zcb);
}

template <int JC>
__global__ void __launch_bounds__(kLineThreads)
    k_bbb_gradlines(const BBCell* __restrict__ cells, const int32_t* __restrict__ order, int kind,
                    const float* __restrict__ target, float contrast, float* __restrict__ loss) {
  const int ci = order[blockIdx.z];
  const BBCell& cc = cells[ci];
  if ((int)blockIdx.x >= cc.gctas) return;
  bb_gradlines<JC>(cc.s, cc.w.z, target ? target + cc.grid_off : nullptr, kind, contrast,
                   cc.w.hdr, cc.w.w2t, cc.w.t2, cc.w.lp, loss ? loss + ci : nullptr, blockIdx.x,
                   cc.gctas);
}

__global__ void k_bbb_ties(const BBCell* __restrict__ cells) {
  const BBCell& cc = cells[blockIdx.z];
  bb_ties(cc.s, cc.w.z, cc.w.hdr, cc.w.w2t, cc.w.t2,
          (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

__global__ void __launch_bounds__(kColThreads) k_bbb_columns(const BBCell* __restrict__ cells) {
  const BBCell& cc = cells[blockIdx.z];
  if ((int)blockIdx.x >= cc.e12) return;
  bb_columns(cc.s, cc.w.q1p, cc.w.w0, cc.w.g0, blockIdx.x);
}

__global__ void k_bbb_gather(const BBCell* __restrict__ cells, const int64_t* __restrict__ bpref,
                             int ncells, int64_t total, const int32_t* __restrict__ band,
                             float2* __restrict__ grad_list) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= total) return;
  const int c = find_cell(bpref, ncells, m);
  const BBCell& cc = cells[c];
  const float2 g = bb_gather(cc.s, band + cc.band_off, m - cc.band_off, cc.w.g0, cc.w.w0,
                             cc.w.w1, cc.w.w2, cc.w.z, cc.w.hdr);
  grad_list[m] = make_float2(g.x * cc.gscale, g.y * cc.gscale);
}

// OR of the cells' status words into *out; the words are cleared.
__global__ void k_bbb_errors(const BBCell* __restrict__ cells, int ncells, int* out) {
  for (int c = threadIdx.x; c < ncells; c += blockDim.x) {
    int* e = &cells[c].w.hdr->err;
    const int v = *e;
    if (v) atomicOr(out, v);
    *e = 0;
  }
}

// Host plan of a batch, kept in dm_bandbox_batch::plan (int64 slots).
constexpr int kBBBMaxZ = 8, kBBBMaxJ = 4;
struct BBBPlan {
  int64_t ncells, total_band;
  int64_t gx[3], gy[3], gz[3];
  int64_t ties_x, col_x, col_smem;
  int64_t nz, zC[kBBBMaxZ], zfirst[kBBBMaxZ], zcount[kBBBMaxZ], zx[kBBBMaxZ], zy[kBBBMaxZ],
      zsmem[kBBBMaxZ];
  int64_t nj, jJC[kBBBMaxJ], jfirst[kBBBMaxJ], jcount[kBBBMaxJ], jx[kBBBMaxJ], jsmem[kBBBMaxJ];
  int64_t off_cells, off_gemm, off_zp, off_zord, off_gord, off_bpref, off_err;
};

// Device-buffer layout of a batch plan for ncells cells.
size_t bbb_desc_layout(int ncells, BBBPlan* p) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += up256(bytes);
    return (int64_t)o;
  };
  const int64_t oc = take(sizeof(BBCell) * ncells);
  const int64_t og = take(sizeof(GemmP) * 3 * (size_t)ncells);
  const int64_t oz = take(sizeof(int32_t) * 3 * (size_t)(ncells + 1));
  const int64_t o1 = take(sizeof(int32_t) * ncells);
  const int64_t o2 = take(sizeof(int32_t) * ncells);
  const int64_t ob = take(sizeof(int64_t) * (size_t)(ncells + 1));
  const int64_t oe = take(sizeof(int));
  if (p) {
    p->off_cells = oc; p->off_gemm = og; p->off_zp = oz; p->off_zord = o1;
    p->off_gord = o2; p->off_bpref = ob; p->off_err = oe;
  }
  return off;
}

template <int C>
cudaError_t zlines_cells(const BBCell* cells, const int32_t* order, unsigned gx, unsigned gy,
                         unsigned gz, size_t smem, float* image, cudaStream_t st) {
  auto k = k_bbb_zlines<C>;
  static std::atomic<bool> done[64];
  cudaError_t e = smem_limit_once(k, done);
  if (e != cudaSuccess) return e;
  k<<<dim3(gx, gy, gz), kLineThreads, smem, st>>>(cells, order, image);
  return cudaGetLastError();
}

template <int JC>
cudaError_t gradlines_cells(const BBCell* cells, const int32_t* order, unsigned gx, unsigned gz,
                            size_t smem, int kind, const float* target, float contrast,
                            float* loss, cudaStream_t st) {
  auto k = k_bbb_gradlines<JC>;
  static std::atomic<bool> done[64];
  cudaError_t e = smem_limit_once(k, done);
  if (e != cudaSuccess) return e;
  k<<<dim3(gx, 1, gz), kLineThreads, smem, st>>>(cells, order, kind, target, contrast, loss);
  return cudaGetLastError();
}

}  // namespace
}  // namespace dm

using namespace dm;

extern "C" {

int dm_band_bounds(const int32_t* band_index, int64_t n_band, const dm_box* box,
                   int32_t* bounds, dm_stream_t stream) {
  if (!box || !bounds || n_band < 0 || (n_band > 0 && !band_index)) return DM_ERR_INVALID_ARG;
  for (int d = 0; d < 3; ++d)
    if (box->shape[d] <= 0) return DM_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  k_bb_bounds_init<<<1, 32, 0, st>>>(bounds);
  if (n_band > 0) {
    const int64_t nb = std::min<int64_t>((n_band + 255) / 256, 1024);
    k_bb_bounds<<<(unsigned)nb, 256, 0, st>>>(band_index, n_band, box->shape[1], box->shape[2],
                                              bounds);
  }
  count_launches(n_band > 0 ? 2 : 1);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

size_t dm_render_loss_bandbox_workspace_size(const dm_box* box, const int32_t bounds[6]) {
  if (!box || !bounds) return 0;
  int32_t lo[3], ext[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = bounds[d];
    ext[d] = bounds[3 + d] - bounds[d] + 1;
  }
  BBShape s;
  if (!make_shape(box->shape, lo, ext, s)) return 0;
  return bb_layout(s, nullptr, nullptr);
}

int dm_render_loss_bandbox_supported(const dm_box* box, const int32_t bounds[6]) {
  if (!box || !bounds) return 0;
  int32_t lo[3], ext[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = bounds[d];
    ext[d] = bounds[3 + d] - bounds[d] + 1;
  }
  BBShape s;
  if (!make_shape(box->shape, lo, ext, s)) return 0;
  if (s.ext[2] > kMaxExt2) return 0;
  if (gradlines_smem(s.n[2], s.ldj) > (size_t)kSmemLimit) return 0;
  if (zlines_smem(s) > (size_t)kSmemLimit) return 0;
  return 1;
}

int dm_render_loss_bandbox(const float* ft_list, const int32_t* band_index, int64_t n_band,
                           const dm_box* box, const int32_t bounds[6], const float* otf,
                           int kind, const float* target, float contrast, float* loss,
                           float* grad_list, float* image, void* workspace, size_t ws_bytes,
                           dm_stream_t stream) {
  if (!box || !bounds || !workspace || !loss || n_band <= 0 || !band_index || !ft_list)
    return DM_ERR_INVALID_ARG;
  if (kind < 0 || kind > 2 || (kind == 1 && !target) || (kind == 2 && grad_list && !target))
    return DM_ERR_INVALID_ARG;
  if (!dm_render_loss_bandbox_supported(box, bounds)) return DM_ERR_UNSUPPORTED;
  if (n_band > (int64_t)INT32_MAX) return DM_ERR_SIZE;
  const size_t need = dm_render_loss_bandbox_workspace_size(box, bounds);
  if (need == 0) return DM_ERR_INVALID_ARG;
  if (ws_bytes < need) return DM_ERR_WORKSPACE;
  int32_t lo[3], ext[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = bounds[d];
    ext[d] = bounds[3 + d] - bounds[d] + 1;
  }
  BBShape s;
  make_shape(box->shape, lo, ext, s);
  BBWs w;
  bb_layout(s, (char*)workspace, &w);
  cudaStream_t st = (cudaStream_t)stream;
  int launches = 0;
  cudaError_t e = cudaSuccess;
  {
    const int64_t tot = (int64_t)s.ext[0] * s.n[0] + (int64_t)s.ext[1] * s.n[1] +
                        (int64_t)s.ext[2] * s.ldw2 + (int64_t)s.n[2] * s.ldj;
    const unsigned nb = (unsigned)std::min<int64_t>((tot + 255) / 256, 1024);
    k_bb_tables<<<nb, 256, 0, st>>>(s, w.w0, w.w1, w.w2, w.w2t, w.hdr);
    ++launches;
  }
  if (cudaMemsetAsync(w.t0, 0, sizeof(float2) * (size_t)s.ext[0] * s.ext[1] * s.ext[2], st) !=
      cudaSuccess)
    return DM_ERR_CUDA;
  k_bb_scatter<<<(unsigned)((n_band + 255) / 256), 256, 0, st>>>(
      s, band_index, n_band, (const float2*)ft_list, otf, w.t0, &w.hdr->err);
  ++launches;
  const int64_t e12 = (int64_t)s.ext[1] * s.ext[2];
  // axis 0: T1[x0][j1 j2] = sum_j0 W0[j0][x0] T0[j0][j1 j2]
  gemm<true>(w.w0, s.n[0], s.n[0], (int)e12, s.ext[0], s.ext[0], w.t0, 0, e12, 1, 0, w.t1, 0,
             e12, 1, 0, 1, st);
  // axis 1: T2[x0][x1][j2] = sum_j1 W1[j1][x1] T1[x0][j1][j2]
  gemm<true>(w.w1, s.n[1], s.n[1], s.ext[2], s.ext[1], s.ext[1], w.t1, e12, s.ext[2], 1, 0,
             w.t2, (int64_t)s.n[1] * s.ext[2], s.ext[2], 1, 0, s.n[0], st);
  launches += 2;
  const float inv_n = (float)(1.0 / (double)s.nvox);
  switch (s.zc) {
    case 1: e = zlines<1>(s, w, inv_n, image, st); break;
    case 2: e = zlines<2>(s, w, inv_n, image, st); break;
    case 3: e = zlines<3>(s, w, inv_n, image, st); break;
    case 4: e = zlines<4>(s, w, inv_n, image, st); break;
    case 5: e = zlines<5>(s, w, inv_n, image, st); break;
    case 6: e = zlines<6>(s, w, inv_n, image, st); break;
    case 7: e = zlines<7>(s, w, inv_n, image, st); break;
    default: e = zlines<8>(s, w, inv_n, image, st); break;
  }
  if (e != cudaSuccess) return DM_ERR_CUDA;
  if (kind == 2 && !grad_list) {  // the image alone
    if (cudaMemsetAsync(loss, 0, sizeof(float), st) != cudaSuccess) return DM_ERR_CUDA;
    count_launches(launches + 1);
    return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
  }
  switch (s.ldj / 8) {
    case 1: e = gradlines<1>(s, w, kind, target, contrast, loss, st); break;
    case 2: e = gradlines<2>(s, w, kind, target, contrast, loss, st); break;
    case 3: e = gradlines<3>(s, w, kind, target, contrast, loss, st); break;
    default: e = gradlines<4>(s, w, kind, target, contrast, loss, st); break;
  }
  if (e != cudaSuccess) return DM_ERR_CUDA;
  launches += 2;
  if (grad_list) {
    k_bb_ties<<<(unsigned)((s.nlines + 127) / 128), 128, 0, st>>>(s, w.z, w.hdr, w.w2t, w.t2);
    // axis 1 (forward), column-major: Q1[kp][j1 j2][x0] = sum_{x1 in split kp} conj(W1[j1][x1]) Q2[x0][x1][j2]
    gemm<false>(w.w1, s.n[1], s.ext[1], s.ext[2], s.n[1], s.q1chunk, w.t2,
                (int64_t)s.n[1] * s.ext[2], s.ext[2], 1, 0, w.q1p, 1,
                (int64_t)s.ext[2] * s.n[0], s.n[0], e12 * s.n[0], s.n[0], st);
    // axis 0 (forward) over the band box, then the band entries
    k_bb_columns<<<(unsigned)e12, kColThreads, sizeof(float2) * (size_t)s.n[0], st>>>(
        s, w.q1p, w.w0, w.g0);
    k_bb_gather<<<(unsigned)((n_band + 255) / 256), 256, 0, st>>>(
        s, band_index, n_band, w.g0, w.w0, w.w1, w.w2, w.z, w.hdr, (float2*)grad_list);
    launches += 4;
  }
  count_launches(launches);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}


// ---------------------------------------------------------------------------
// Batches of boxes (one plan, one workspace; see the header).

size_t dm_bandbox_batch_desc_size(int ncells) {
  return ncells > 0 ? bbb_desc_layout(ncells, nullptr) : 0;
}

static int bbb_shapes(const dm_cell* cells, const int32_t* bounds, int ncells,
                      std::vector<BBShape>& shapes, size_t* ws_total) {
  if (!cells || !bounds || ncells <= 0) return DM_ERR_INVALID_ARG;
  shapes.resize(ncells);
  size_t tot = 0;
  for (int i = 0; i < ncells; ++i) {
    if (cells[i].n_band <= 0) return DM_ERR_INVALID_ARG;
    if (!dm_render_loss_bandbox_supported(&cells[i].box, bounds + 6 * i)) return DM_ERR_UNSUPPORTED;
    int32_t lo[3], ext[3];
    for (int d = 0; d < 3; ++d) {
      lo[d] = bounds[6 * i + d];
      ext[d] = bounds[6 * i + 3 + d] - bounds[6 * i + d] + 1;
    }
    if (!make_shape(cells[i].box.shape, lo, ext, shapes[i])) return DM_ERR_UNSUPPORTED;
    // the batch's (cell x position) entries already fill the GPU: the axis-1 forward
    // contraction runs over all positions in one block instead of K splits
    shapes[i].q1split = 1;
    shapes[i].q1chunk = (shapes[i].n[1] + 15) / 16 * 16;
    tot += bb_layout(shapes[i], nullptr, nullptr);
  }
  *ws_total = tot;
  return DM_OK;
}

int dm_bandbox_batch_workspace_size(const dm_cell* cells, const int32_t* bounds, int ncells,
                                    size_t* bytes) {
  if (!bytes) return DM_ERR_INVALID_ARG;
  std::vector<BBShape> shapes;
  size_t tot = 0;
  const int r = bbb_shapes(cells, bounds, ncells, shapes, &tot);
  *bytes = r == DM_OK ? tot : 0;
  return r;
}

int dm_bandbox_batch_plan(const dm_cell* cells, const int32_t* bounds, int ncells, void* desc,
                          size_t desc_bytes, void* workspace, size_t ws_bytes,
                          dm_bandbox_batch* out, dm_stream_t stream) {
  static_assert(sizeof(BBBPlan) <= sizeof(((dm_bandbox_batch*)nullptr)->plan), "plan slots");
  if (!desc || !workspace || !out) return DM_ERR_INVALID_ARG;
  std::vector<BBShape> sh;
  size_t need = 0;
  int r = bbb_shapes(cells, bounds, ncells, sh, &need);
  if (r != DM_OK) return r;
  if (ws_bytes < need) return DM_ERR_WORKSPACE;
  BBBPlan P;
  memset(&P, 0, sizeof(P));
  const size_t dbytes = bbb_desc_layout(ncells, &P);
  if (desc_bytes < dbytes) return DM_ERR_WORKSPACE;
  std::vector<char> host(dbytes, 0);
  BBCell* hc = (BBCell*)(host.data() + P.off_cells);
  GemmP* hg = (GemmP*)(host.data() + P.off_gemm);
  int32_t* hz = (int32_t*)(host.data() + P.off_zp);
  int32_t* zord = (int32_t*)(host.data() + P.off_zord);
  int32_t* gord = (int32_t*)(host.data() + P.off_gord);
  int64_t* bpref = (int64_t*)(host.data() + P.off_bpref);
  const int sms = num_sms();
  size_t off = 0;
  bpref[0] = 0;
  for (int k = 0; k < 3; ++k) hz[k * (ncells + 1)] = 0;
  P.ncells = ncells;
  for (int i = 0; i < ncells; ++i) {
    const BBShape& s = sh[i];
    BBCell& c = hc[i];
    c.s = s;
    off += bb_layout(s, (char*)workspace + off, &c.w);
    c.band_off = bpref[i];
    c.nband = cells[i].n_band;
    bpref[i + 1] = bpref[i] + c.nband;
    c.grid_off = cells[i].grid_offset;
    c.inv_n = (float)(1.0 / (double)s.nvox);
    c.gscale = c.inv_n;
    c.zcb = (int32_t)(s.ldw2 / (32 * s.zc));
    c.e12 = s.ext[1] * s.ext[2];
    const int64_t e12 = c.e12;
    GemmP g[3];
    g[0] = gemm_p(c.w.w0, s.n[0], s.n[0], (int)e12, s.ext[0], s.ext[0], c.w.t0, 0, e12, 1, 0,
                  c.w.t1, 0, e12, 1, 0, 1);
    g[1] = gemm_p(c.w.w1, s.n[1], s.n[1], s.ext[2], s.ext[1], s.ext[1], c.w.t1, e12, s.ext[2], 1,
                  0, c.w.t2, (int64_t)s.n[1] * s.ext[2], s.ext[2], 1, 0, s.n[0]);
    g[2] = gemm_p(c.w.w1, s.n[1], s.ext[1], s.ext[2], s.n[1], s.q1chunk, c.w.t2,
                  (int64_t)s.n[1] * s.ext[2], s.ext[2], 1, 0, c.w.q1p, 1,
                  (int64_t)s.ext[2] * s.n[0], s.n[0], e12 * s.n[0], s.n[0]);
    for (int k = 0; k < 3; ++k) {
      hg[k * ncells + i] = g[k];
      const dim3 gd = gemm_grid(g[k], k == 2 ? 2 : 4);
      P.gx[k] = std::max<int64_t>(P.gx[k], gd.x);
      P.gy[k] = std::max<int64_t>(P.gy[k], gd.y);
      hz[k * (ncells + 1) + i + 1] = hz[k * (ncells + 1) + i] + (int32_t)gd.z;
    }
    P.ties_x = std::max<int64_t>(P.ties_x, (s.nlines + 127) / 128);
    P.col_x = std::max<int64_t>(P.col_x, e12);
    P.col_smem = std::max<int64_t>(P.col_smem, (int64_t)sizeof(float2) * s.n[0]);
  }
  P.total_band = bpref[ncells];
  for (int k = 0; k < 3; ++k) {
    P.gz[k] = hz[k * (ncells + 1) + ncells];
    if (P.gz[k] > 65535 || P.gy[k] > 65535) return DM_ERR_SIZE;
  }
  if (P.ties_x > INT32_MAX || P.col_x > INT32_MAX) return DM_ERR_SIZE;
  // z pass groups (by columns per thread), gradient pass groups (by offset groups)
  std::vector<int> idx(ncells);
  for (int i = 0; i < ncells; ++i) idx[i] = i;
  auto jc_of = [&](int i) { return std::min(4, sh[i].ldj / 8); };
  // CTAs of a line-pass launch: about two per SM (per column block), shared by the
  // launch's cells in proportion to their work (voxels x band extent), at least one
  // and at most one per line tile
  // (as many as shared memory lets reside, up to four, when the launch's tiles are
  // small)
  auto share = [&](int first, int count, const std::vector<int>& ord, bool z) {
    double wsum = 0.0;
    size_t smem = 0;
    for (int k = first; k < first + count; ++k) {
      const BBShape& s = sh[ord[k]];
      wsum += (double)s.nvox * s.ext[2];
      smem = std::max(smem, z ? zlines_smem(s) : gradlines_smem(s.n[2], s.ldj));
    }
    const int per_sm = (int)std::max<size_t>(
        2, std::min<size_t>(4, (size_t)kSmemLimit / std::max<size_t>(smem + 8192, 1)));
    for (int k = first; k < first + count; ++k) {
      const BBShape& s = sh[ord[k]];
      const int64_t tiles = (s.nlines + kLines - 1) / kLines;
      const double w = (double)per_sm * sms * ((double)s.nvox * s.ext[2]) / wsum;
      const int32_t ctas =
          (int32_t)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)(w + 0.5)));
      if (z) hc[ord[k]].zctas = ctas; else hc[ord[k]].gctas = ctas;
    }
  };
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return sh[a].zc < sh[b].zc; });
  for (int k0 = 0; k0 < ncells;) {
    int k1 = k0;
    while (k1 < ncells && sh[idx[k1]].zc == sh[idx[k0]].zc) ++k1;
    share(k0, k1 - k0, idx, true);
    k0 = k1;
  }
  for (int k = 0; k < ncells;) {
    const int C = sh[idx[k]].zc;
    const int g = (int)P.nz++;
    if (g >= kBBBMaxZ) return DM_ERR_SIZE;
    P.zC[g] = C;
    P.zfirst[g] = k;
    for (; k < ncells && sh[idx[k]].zc == C; ++k) {
      zord[k] = idx[k];
      P.zcount[g] += 1;
      P.zx[g] = std::max<int64_t>(P.zx[g], hc[idx[k]].zctas);
      P.zy[g] = std::max<int64_t>(P.zy[g], hc[idx[k]].zcb);
      P.zsmem[g] = std::max<int64_t>(P.zsmem[g], (int64_t)zlines_smem(sh[idx[k]]));
    }
  }
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return jc_of(a) < jc_of(b); });
  for (int k0 = 0; k0 < ncells;) {
    int k1 = k0;
    while (k1 < ncells && jc_of(idx[k1]) == jc_of(idx[k0])) ++k1;
    share(k0, k1 - k0, idx, false);
    k0 = k1;
  }
  for (int k = 0; k < ncells;) {
    const int J = jc_of(idx[k]);
    const int g = (int)P.nj++;
    if (g >= kBBBMaxJ) return DM_ERR_SIZE;
    P.jJC[g] = J;
    P.jfirst[g] = k;
    for (; k < ncells && jc_of(idx[k]) == J; ++k) {
      gord[k] = idx[k];
      P.jcount[g] += 1;
      P.jx[g] = std::max<int64_t>(P.jx[g], hc[idx[k]].gctas);
      P.jsmem[g] = std::max<int64_t>(
          P.jsmem[g], (int64_t)gradlines_smem(sh[idx[k]].n[2], sh[idx[k]].ldj));
    }
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemcpyAsync(desc, host.data(), dbytes, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return DM_ERR_CUDA;
  // zero band boxes (only the band voxels are ever written), counters and status
  // words, then the root tables of every cell
  if (cudaMemsetAsync(workspace, 0, need, st) != cudaSuccess) return DM_ERR_CUDA;
  for (int i = 0; i < ncells; ++i) {
    const BBShape& s = sh[i];
    const BBWs& w = hc[i].w;
    const int64_t tot = (int64_t)s.ext[0] * s.n[0] + (int64_t)s.ext[1] * s.n[1] +
                        (int64_t)s.ext[2] * s.ldw2 + (int64_t)s.n[2] * s.ldj;
    const unsigned nb = (unsigned)std::min<int64_t>((tot + 255) / 256, 1024);
    k_bb_tables<<<nb, 256, 0, st>>>(s, w.w0, w.w1, w.w2, w.w2t, w.hdr);
  }
  count_launches(ncells);
  if (cudaStreamSynchronize(st) != cudaSuccess) return DM_ERR_CUDA;
  memset(out, 0, sizeof(*out));
  out->ncells = ncells;
  out->workspace_bytes = (int64_t)need;
  memcpy(out->plan, &P, sizeof(P));
  out->cells = desc;
  out->workspace = workspace;
  return DM_OK;
}

int dm_bandbox_batch_render_loss(const dm_bandbox_batch* bb, const float* ft_list,
                                 const int32_t* band_index, const float* otf, int kind,
                                 const float* target, float contrast, float* loss,
                                 float* grad_list, float* image, dm_stream_t stream) {
  if (!bb || !bb->cells || !ft_list || !band_index || !loss) return DM_ERR_INVALID_ARG;
  if ((kind != 0 && kind != 1) || (kind == 1 && !target)) return DM_ERR_INVALID_ARG;
  BBBPlan P;
  memcpy(&P, bb->plan, sizeof(P));
  const int n = (int)P.ncells;
  if (n <= 0 || n != bb->ncells) return DM_ERR_INVALID_ARG;
  const char* d = (const char*)bb->cells;
  const BBCell* cells = (const BBCell*)(d + P.off_cells);
  const GemmP* gp = (const GemmP*)(d + P.off_gemm);
  const int32_t* zp = (const int32_t*)(d + P.off_zp);
  const int32_t* zord = (const int32_t*)(d + P.off_zord);
  const int32_t* gord = (const int32_t*)(d + P.off_gord);
  const int64_t* bpref = (const int64_t*)(d + P.off_bpref);
  cudaStream_t st = (cudaStream_t)stream;
  int launches = 0;
  const unsigned nbb = (unsigned)((P.total_band + 255) / 256);
  k_bbb_scatter<<<nbb, 256, 0, st>>>(cells, bpref, n, P.total_band, band_index,
                                      (const float2*)ft_list, otf);
  k_bbb_gemm<true><<<dim3((unsigned)P.gx[0], (unsigned)P.gy[0], (unsigned)P.gz[0]),
                     kGemmThreads, 0, st>>>(gp, zp, n);
  k_bbb_gemm<true><<<dim3((unsigned)P.gx[1], (unsigned)P.gy[1], (unsigned)P.gz[1]),
                     kGemmThreads, 0, st>>>(gp + n, zp + (n + 1), n);
  launches += 3;
  cudaError_t e = cudaSuccess;
  for (int g = 0; g < P.nz && e == cudaSuccess; ++g) {
    const int32_t* ord = zord + P.zfirst[g];
    const unsigned gx = (unsigned)P.zx[g], gy = (unsigned)P.zy[g], gz = (unsigned)P.zcount[g];
    const size_t sm = (size_t)P.zsmem[g];
    switch (P.zC[g]) {
      case 1: e = zlines_cells<1>(cells, ord, gx, gy, gz, sm, image, st); break;
      case 2: e = zlines_cells<2>(cells, ord, gx, gy, gz, sm, image, st); break;
      case 3: e = zlines_cells<3>(cells, ord, gx, gy, gz, sm, image, st); break;
      case 4: e = zlines_cells<4>(cells, ord, gx, gy, gz, sm, image, st); break;
      case 5: e = zlines_cells<5>(cells, ord, gx, gy, gz, sm, image, st); break;
      case 6: e = zlines_cells<6>(cells, ord, gx, gy, gz, sm, image, st); break;
      case 7: e = zlines_cells<7>(cells, ord, gx, gy, gz, sm, image, st); break;
      default: e = zlines_cells<8>(cells, ord, gx, gy, gz, sm, image, st); break;
    }
    ++launches;
  }
  for (int g = 0; g < P.nj && e == cudaSuccess; ++g) {
    const int32_t* ord = gord + P.jfirst[g];
    const unsigned gx = (unsigned)P.jx[g], gz = (unsigned)P.jcount[g];
    const size_t sm = (size_t)P.jsmem[g];
    switch (P.jJC[g]) {
      case 1: e = gradlines_cells<1>(cells, ord, gx, gz, sm, kind, target, contrast, loss, st); break;
      case 2: e = gradlines_cells<2>(cells, ord, gx, gz, sm, kind, target, contrast, loss, st); break;
      case 3: e = gradlines_cells<3>(cells, ord, gx, gz, sm, kind, target, contrast, loss, st); break;
      default: e = gradlines_cells<4>(cells, ord, gx, gz, sm, kind, target, contrast, loss, st); break;
    }
    ++launches;
  }
  if (e != cudaSuccess) return DM_ERR_CUDA;
  if (grad_list) {
    k_bbb_ties<<<dim3((unsigned)P.ties_x, 1, (unsigned)n), 128, 0, st>>>(cells);
    k_bbb_gemm<false><<<dim3((unsigned)P.gx[2], (unsigned)P.gy[2], (unsigned)P.gz[2]),
                        kGemmThreads, 0, st>>>(gp + 2 * n, zp + 2 * (n + 1), n);
    k_bbb_columns<<<dim3((unsigned)P.col_x, 1, (unsigned)n), kColThreads, (size_t)P.col_smem,
                    st>>>(cells);
    k_bbb_gather<<<nbb, 256, 0, st>>>(cells, bpref, n, P.total_band, band_index,
                                       (float2*)grad_list);
    launches += 4;
  }
  count_launches(launches);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

int dm_bandbox_batch_device_error(const dm_bandbox_batch* bb, int* out_flags, dm_stream_t stream) {
  if (!bb || !bb->cells || !out_flags) return DM_ERR_INVALID_ARG;
  BBBPlan P;
  memcpy(&P, bb->plan, sizeof(P));
  int* slot = (int*)((char*)bb->cells + P.off_err);
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemsetAsync(slot, 0, sizeof(int), st) != cudaSuccess) return DM_ERR_CUDA;
  k_bbb_errors<<<1, 256, 0, st>>>((const BBCell*)((const char*)bb->cells + P.off_cells),
                                  (int)P.ncells, slot);
  count_launches(1);
  int v = 0;
  if (cudaMemcpyAsync(&v, slot, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return DM_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return DM_ERR_CUDA;
  *out_flags = v;
  return DM_OK;
}

}  // extern "C"
