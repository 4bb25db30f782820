// meshFT forward / backward for sm_100a: face records, epilogues, the adjoint's
// face order, the vertex <- face CSR, and the launch plans.  The main kernels
// (k_meshft_fwd, k_meshft_bwd) and their work decomposition are in
// meshft_kernels.cuh.  Partial sums go to HBM and are reduced in a fixed order
// (deterministic, no atomics); a CSR gather sums face contributions per vertex
// in a fixed order.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <string.h>

#include <algorithm>
#include <atomic>

#include "dm_common.cuh"
#include "meshft_internal.h"
#include "meshft_kernels.cuh"
#include "pair_math.cuh"

namespace dm {

constexpr int64_t kSortMinFaces = 1024;  // adjoint face order by size from this many faces

// ---------------------------------------------------------------------------
// Face records and per-block sums of area * coeff (replaces the host loops of
// fourier3d_cuda_kernel.cu:16-51).

__global__ void k_face_prep(Cells cells, const float* __restrict__ verts,
                            const int64_t* __restrict__ faces, const float* __restrict__ coeff,
                            FaceRec* __restrict__ recs, double* __restrict__ area_part, int* err) {
  __shared__ double sh[40];
  const int ci = cell_find(cells, blockIdx.x, [](const CellDesc& d) { return d.face_blk0; });
  const CellDesc d = cell_get(cells, ci);
  const int f = (blockIdx.x - d.face_blk0) * kBlk + threadIdx.x;
  double ac = 0.0;
  if (f < d.nt) {
    const int64_t gf = d.f_off + f;
    int64_t iv[3];
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      iv[k] = faces[3 * gf + k];
      if (iv[k] < 0 || iv[k] >= d.nv) {
        ok = false;
        iv[k] = 0;
      }
    }
    if (!ok) set_error(err, DM_ERR_BAD_INDEX);
    double p[3][3];
    bool fin = true;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        p[k][j] = (double)verts[3 * (d.v_off + iv[k]) + j];
        if (!isfinite(p[k][j])) {  // reported; the face is evaluated at lo instead
          fin = false;
          p[k][j] = d.lo[j];
        }
      }
    if (!fin) set_error(err, DM_ERR_NONFINITE);
    FaceRec r;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double sc = 2147483648.0 / d.len[j];
      r.Ua[j] = (uint32_t)(long long)llrint((p[0][j] - d.lo[j]) * sc);
      r.Ub[j] = (uint32_t)(long long)llrint((p[1][j] - d.lo[j]) * sc);
      r.Uc[j] = (uint32_t)(long long)llrint((p[2][j] - d.lo[j]) * sc);
      const double hs = 1.5707963267948966 / d.len[j];
      r.hab[j] = (float)((p[1][j] - p[0][j]) * hs);
      r.hbc[j] = (float)((p[2][j] - p[1][j]) * hs);
    }
    const double e1[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
    const double e2[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
    const double cx = e1[1] * e2[2] - e1[2] * e2[1];
    const double cy = e1[2] * e2[0] - e1[0] * e2[2];
    const double cz = e1[0] * e2[1] - e1[1] * e2[0];
    ac = 0.5 * sqrt(cx * cx + cy * cy + cz * cz) * (coeff ? (double)coeff[gf] : 1.0);
    r.area_coeff = (float)ac;
    recs[gf] = r;
  }
  const double s = block_sum_d(ac, sh);
  if (threadIdx.x == 0) area_part[blockIdx.x] = s;
}


// ft_list = (2/M) * sum over splits; optional scatter of ft * OTF into the grid.
// With a mirrored band (herm) the entries past ne are conj of their mirrors.
__global__ void k_meshft_fwd_epi(Cells cells, const int32_t* __restrict__ band_index,
                                 const float2* __restrict__ fpart,
                                 const double* __restrict__ area_part,
                                 const float* __restrict__ otf, float2* __restrict__ ft_list,
                                 float2* __restrict__ grid, int* err) {
  __shared__ double sh[40];
  const int ci = cell_find(cells, blockIdx.x, [](const CellDesc& d) { return d.band_blk0; });
  const CellDesc d = cell_get(cells, ci);
  const double M = block_sum_list(area_part + d.face_blk0, (d.nt + kBlk - 1) / kBlk, sh);
  const int m = (blockIdx.x - d.band_blk0) * kBlk + threadIdx.x;
  if (m >= d.ne) return;
  double sx = 0.0, sy = 0.0;
  const float2* p = fpart + d.fpart_off + m;
  // eight loads in flight, summed in split order (fixed result)
  int s = 0;
  for (; s + 8 <= d.fsplit; s += 8) {
    float2 v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = p[(int64_t)(s + u) * d.ne];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      sx += v[u].x;
      sy += v[u].y;
    }
  }
  for (; s < d.fsplit; ++s) {
    const float2 v = p[(int64_t)s * d.ne];
    sx += v.x;
    sy += v.y;
  }
  const double sc = d.nt > 0 ? 2.0 / M : 0.0;  // no faces: ft = 0 as in the reference
  const float2 ft = make_float2((float)(sx * sc), (float)(sy * sc));
  const int64_t nvox = (int64_t)d.n[0] * d.n[1] * d.n[2];
  const int mr = d.nband - 1 - m;  // mirror entry
  const bool mirror = d.herm && mr != m;
  ft_list[d.b_off + m] = ft;
  if (mirror) ft_list[d.b_off + mr] = make_float2(ft.x, -ft.y);
  const int32_t idx = band_index[d.b_off + m];
  const int32_t idr = mirror ? band_index[d.b_off + mr] : idx;
  const bool ok = idx >= 0 && (int64_t)idx < nvox &&
                  (!mirror || (int64_t)idr == nvox - 1 - (int64_t)idx);
  if (!ok) {
    set_error(err, DM_ERR_BAD_INDEX);
    return;
  }
  if (grid) {
    const float o = otf ? otf[d.grid_off + idx] : 1.0f;
    grid[d.grid_off + idx] = make_float2(ft.x * o, ft.y * o);
    if (mirror) {
      const float orr = otf ? otf[d.grid_off + idr] : 1.0f;
      grid[d.grid_off + idr] = make_float2(ft.x * orr, -ft.y * orr);
    }
  }
}

// ---------------------------------------------------------------------------
// Backward: band records with the cotangent, and per-block sums of
// s = sum Re(conj(g) ft) over the whole band.  With a mirrored band (herm) the
// record of entry m < ne carries g(xi) + conj(g(-xi)): the adjoint of
// ft(-xi) = conj(ft(xi)).

__global__ void k_bwd_band_prep(Cells cells, const int32_t* __restrict__ band_index,
                                const float2* __restrict__ grad_list,
                                const float2* __restrict__ grad_grid,
                                const float* __restrict__ otf, float grad_scale,
                                const float2* __restrict__ ft_list, XiRec* __restrict__ xrec,
                                float* __restrict__ grad_otf_band, double* __restrict__ s_part,
                                int* err) {
  __shared__ double sh[40];
  const int ci = cell_find(cells, blockIdx.x, [](const CellDesc& d) { return d.band_blk0; });
  const CellDesc d = cell_get(cells, ci);
  const int m = (blockIdx.x - d.band_blk0) * kBlk + threadIdx.x;
  const int64_t nvox = (int64_t)d.n[0] * d.n[1] * d.n[2];
  double s = 0.0;
  if (m < d.nband) {
    const int64_t gm = d.b_off + m;
    int32_t idx = band_index[gm];
    const bool ok = idx >= 0 && (int64_t)idx < nvox;
    if (!ok) {
      set_error(err, DM_ERR_BAD_INDEX);
      idx = 0;
    }
    float2 G;
    float2 g = band_cotangent(d, gm, idx, ok, grad_list, grad_grid, otf, grad_scale, G);
    const float2 ft = ft_list[gm];
    if (grad_otf_band) grad_otf_band[gm] = grad_scale * (G.x * ft.x + G.y * ft.y);
    s = (double)g.x * ft.x + (double)g.y * ft.y;
    if (m < d.ne) {
      const int mr = d.nband - 1 - m;
      if (d.herm && mr != m) {
        const int64_t gr = d.b_off + mr;
        int32_t idr = band_index[gr];
        const bool okr = ok && (int64_t)idr == nvox - 1 - (int64_t)idx;
        if (!okr) {
          set_error(err, DM_ERR_BAD_INDEX);
          idr = 0;
        }
        float2 Gr;
        const float2 gr_ = band_cotangent(d, gr, idr, okr, grad_list, grad_grid, otf,
                                          grad_scale, Gr);
        g.x += gr_.x;
        g.y -= gr_.y;
      }
      XiRec r;
      band_to_m(idx, d, r.mi);
#pragma unroll
      for (int k = 0; k < 3; ++k) r.mf[k] = (float)r.mi[k];
      r.g_re = g.x;
      r.g_im = g.y;
      xrec[gm] = r;
    }
  }
  const double t = block_sum_d(s, sh);
  if (threadIdx.x == 0) s_part[blockIdx.x] = t;
}


// Per-face epilogue: reduce chunks, then
//   contrib[f][v][j] = trisar * (pi/L_j) * Q[v][j] + (c/M)(2r - s) dA/dv_j
//   grad_coeff[f]    = (A/M)(2r - s)
// (vertex adjoint of fourier3d_cuda_kernel.cu:365-394 with w and gradmeshar of
// .cu:26-32 folded per face; Faces_coeff gradient from trisar = 2Ac/M).
__global__ void k_bwd_face_epi(Cells cells, const float* __restrict__ verts,
                               const int64_t* __restrict__ faces,
                               const float* __restrict__ coeff,
                               const double* __restrict__ area_part,
                               const double* __restrict__ s_part,
                               const float* __restrict__ bpart, const int32_t* __restrict__ slot_of,
                               float* __restrict__ contrib, float* __restrict__ grad_coeff) {
  __shared__ double sh[40];
  const int ci = cell_find(cells, blockIdx.x, [](const CellDesc& d) { return d.face_blk0; });
  const CellDesc d = cell_get(cells, ci);
  const double M = block_sum_list(area_part + d.face_blk0, (d.nt + kBlk - 1) / kBlk, sh);
  const double S = block_sum_list(s_part + d.band_blk0, (d.nband + kBlk - 1) / kBlk, sh);
  const int f = (blockIdx.x - d.face_blk0) * kBlk + threadIdx.x;
  if (f >= d.nt) return;
  const int64_t gf = d.f_off + f;
  double q[10];
#pragma unroll
  for (int i = 0; i < 10; ++i) q[i] = 0.0;
  const float* p = bpart + d.bpart_off + (slot_of ? (int64_t)slot_of[gf] - d.f_off : f);
  for (int c = 0; c < d.bchunks; ++c) {
#pragma unroll
    for (int i = 0; i < 10; ++i) q[i] += p[((int64_t)c * 10 + i) * d.nt];
  }
  int64_t iv[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    iv[k] = faces[3 * gf + k];
    if (iv[k] < 0 || iv[k] >= d.nv) iv[k] = 0;
  }
  double P[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int j = 0; j < 3; ++j) P[k][j] = (double)verts[3 * (d.v_off + iv[k]) + j];
  const double e1[3] = {P[1][0] - P[0][0], P[1][1] - P[0][1], P[1][2] - P[0][2]};
  const double e2[3] = {P[2][0] - P[0][0], P[2][1] - P[0][1], P[2][2] - P[0][2]};
  double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                 e1[0] * e2[1] - e1[1] * e2[0]};
  const double nn = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  const double A = 0.5 * nn;
  n[0] /= nn;
  n[1] /= nn;
  n[2] /= nn;
  const double c = (double)coeff[gf];
  const double trisar = 2.0 * A * c / M;
  const double k2 = 2.0 * q[9] - S;
  const double kk = (c / M) * k2;
  if (grad_coeff) grad_coeff[gf] = (float)((A / M) * k2);
  // dA/dv = n x (opposite edge, taken cyclically) / 2
  const int nxt[3] = {1, 2, 0}, prv[3] = {2, 0, 1};
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    const double* pn = P[nxt[v]];
    const double* pp = P[prv[v]];
    const double e[3] = {pp[0] - pn[0], pp[1] - pn[1], pp[2] - pn[2]};  // for a: c - b
    const double dA[3] = {0.5 * (n[1] * e[2] - n[2] * e[1]), 0.5 * (n[2] * e[0] - n[0] * e[2]),
                          0.5 * (n[0] * e[1] - n[1] * e[0])};
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double xs = 3.141592653589793 / d.len[j];
      contrib[9 * gf + 3 * v + j] = (float)(trisar * xs * q[3 * v + j] + kk * dA[j]);
    }
  }
}

// grad_verts[v] = sum over the CSR entries of v (fixed order) of contrib.
__global__ void k_vertex_gather(int64_t nv_total, const int32_t* __restrict__ off,
                                const int32_t* __restrict__ ent,
                                const float* __restrict__ contrib, float* __restrict__ grad_verts) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv_total) return;
  float g0 = 0.f, g1 = 0.f, g2 = 0.f;
  const int32_t b = off[v], e = off[v + 1];
  for (int32_t i = b; i < e; ++i) {
    const int32_t x = ent[i];
    const float* c = contrib + 9 * (int64_t)(x / 3) + 3 * (x % 3);
    g0 += c[0];
    g1 += c[1];
    g2 += c[2];
  }
  grad_verts[3 * v + 0] = g0;
  grad_verts[3 * v + 1] = g1;
  grad_verts[3 * v + 2] = g2;
}

// ---------------------------------------------------------------------------
// Face order for the adjoint: faces of each cell sorted by size (a stable
// counting sort on 8 buckets per octave of the longest edge, in phase units).
// In the adjoint a warp's lanes are faces at the same frequency; whether a pair
// takes the series or the pivot path depends on the face's size, so a mesh whose
// face sizes spread (a fit that crumples the surface) splits most warps over
// both paths unless similar faces share a warp.  Slot f of a cell then holds face
// order[f]; slot_of is the inverse.  Per-face sums keep their order, so only the
// warp-uniform choice of the series coefficient set can change (both sets agree
// to their truncation error).

constexpr int kKeyBins = 256;

__device__ __forceinline__ int face_size_key(const FaceRec& r) {
  const float ab = r.hab[0] * r.hab[0] + r.hab[1] * r.hab[1] + r.hab[2] * r.hab[2];
  const float bc = r.hbc[0] * r.hbc[0] + r.hbc[1] * r.hbc[1] + r.hbc[2] * r.hbc[2];
  const float c0 = r.hab[0] + r.hbc[0], c1 = r.hab[1] + r.hbc[1], c2 = r.hab[2] + r.hbc[2];
  const float ca = c0 * c0 + c1 * c1 + c2 * c2;
  const float m = fmaxf(ab, fmaxf(bc, ca));
  if (!(m > 0.f)) return 0;
  const int k = (int)floorf(4.0f * log2f(m)) + kKeyBins / 2;  // 8 bins per octave of length
  return min(max(k, 0), kKeyBins - 1);
}

// Per face block (the 256-face blocks of k_face_prep): key histogram.
__global__ void k_face_key_hist(Cells cells, const FaceRec* __restrict__ recs,
                                int32_t* __restrict__ hist) {
  __shared__ int32_t h[kKeyBins];
  const int ci = cell_find(cells, blockIdx.x, [](const CellDesc& d) { return d.face_blk0; });
  const CellDesc d = cell_get(cells, ci);
  h[threadIdx.x] = 0;
  __syncthreads();
  const int f = (blockIdx.x - d.face_blk0) * kBlk + threadIdx.x;
  if (f < d.nt) atomicAdd(&h[face_size_key(recs[d.f_off + f])], 1);
  __syncthreads();
  hist[(int64_t)blockIdx.x * kKeyBins + threadIdx.x] = h[threadIdx.x];
}

// One CTA per cell (thread = bin): first slot of every (block, bin).
__global__ void k_face_key_scan(Cells cells, const int32_t* __restrict__ hist,
                                int32_t* __restrict__ first) {
  __shared__ int32_t wsum[kKeyBins / 32];
  const CellDesc d = cell_get(cells, blockIdx.x);
  const int nblk = (d.nt + kBlk - 1) / kBlk;
  const int k = threadIdx.x, lane = k & 31, warp = k >> 5;
  int32_t sum = 0;
#pragma unroll 8
  for (int b = 0; b < nblk; ++b) sum += hist[(int64_t)(d.face_blk0 + b) * kKeyBins + k];
  // exclusive scan over the bins (one bin per thread): warp scans, then the warp totals
  int32_t inc = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t n = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += n;
  }
  if (lane == 31) wsum[warp] = inc;
  __syncthreads();
  int32_t before = 0;
#pragma unroll
  for (int w = 0; w < kKeyBins / 32; ++w) before += w < warp ? wsum[w] : 0;
  int32_t run = (int32_t)d.f_off + before + inc - sum;
#pragma unroll 8
  for (int b = 0; b < nblk; ++b) {
    const int64_t o = (int64_t)(d.face_blk0 + b) * kKeyBins + k;
    first[o] = run;
    run += hist[o];
  }
}

// Per face block: stable slots (warps in order, lanes in order within a key).
__global__ void k_face_key_scatter(Cells cells, const FaceRec* __restrict__ recs,
                                   const int32_t* __restrict__ first, int32_t* __restrict__ order,
                                   int32_t* __restrict__ slot_of) {
  __shared__ int32_t base[kKeyBins];
  const int ci = cell_find(cells, blockIdx.x, [](const CellDesc& d) { return d.face_blk0; });
  const CellDesc d = cell_get(cells, ci);
  base[threadIdx.x] = first[(int64_t)blockIdx.x * kKeyBins + threadIdx.x];
  __syncthreads();
  const int f = (blockIdx.x - d.face_blk0) * kBlk + threadIdx.x;
  const bool live = f < d.nt;
  const int key = live ? face_size_key(recs[d.f_off + f]) : -1 - (int)(threadIdx.x & 31);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned same = __match_any_sync(0xffffffffu, key);
  const int rank = __popc(same & ((1u << lane) - 1u));
  for (int w = 0; w < kBlk / 32; ++w) {
    if (warp == w && live) {
      const int32_t slot = base[key] + rank;
      order[slot] = (int32_t)(d.f_off + f);
      slot_of[d.f_off + f] = slot;
    }
    __syncthreads();
    if (warp == w && live && rank == 0) base[key] += __popc(same);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Topology: vertex <- face CSR over the concatenated mesh of a launch.

__global__ void k_csr_count(Cells cells, const int64_t* __restrict__ faces,
                            int32_t* __restrict__ count, int* err) {
  const int ci = cell_find(cells, blockIdx.x, [](const CellDesc& d) { return d.face_blk0; });
  const CellDesc d = cell_get(cells, ci);
  const int f = (blockIdx.x - d.face_blk0) * kBlk + threadIdx.x;
  if (f >= d.nt) return;
  const int64_t gf = d.f_off + f;
  for (int k = 0; k < 3; ++k) {
    const int64_t v = faces[3 * gf + k];
    if (v < 0 || v >= d.nv) {
      set_error(err, DM_ERR_BAD_INDEX);
      continue;
    }
    atomicAdd(&count[d.v_off + v], 1);
  }
}

// Exclusive scan of count[0..n) into off[0..n] by one block.
__global__ void k_csr_scan(const int32_t* __restrict__ count, int32_t* __restrict__ off,
                           int64_t n) {
  __shared__ int32_t sh[1024];
  const int T = blockDim.x;
  const int64_t per = (n + T - 1) / T;
  const int64_t b = threadIdx.x * per, e = (b + per < n) ? b + per : n;
  int32_t s = 0;
  for (int64_t i = b; i < e; ++i) s += count[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < T; o <<= 1) {
    int32_t v = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += v;
    __syncthreads();
  }
  int32_t run = sh[threadIdx.x] - s;
  for (int64_t i = b; i < e; ++i) {
    off[i] = run;
    run += count[i];
  }
  if (threadIdx.x == T - 1) off[n] = sh[T - 1];
}

__global__ void k_csr_fill(Cells cells, const int64_t* __restrict__ faces,
                           const int32_t* __restrict__ off, int32_t* __restrict__ cursor,
                           int32_t* __restrict__ ent) {
  const int ci = cell_find(cells, blockIdx.x, [](const CellDesc& d) { return d.face_blk0; });
  const CellDesc d = cell_get(cells, ci);
  const int f = (blockIdx.x - d.face_blk0) * kBlk + threadIdx.x;
  if (f >= d.nt) return;
  const int64_t gf = d.f_off + f;
  for (int k = 0; k < 3; ++k) {
    const int64_t v = faces[3 * gf + k];
    if (v < 0 || v >= d.nv) continue;
    const int64_t gv = d.v_off + v;
    const int32_t pos = off[gv] + atomicAdd(&cursor[gv], 1);
    ent[pos] = (int32_t)(3 * gf + k);
  }
}

// Insertion-sort each vertex's entries: a fixed summation order per vertex.
__global__ void k_csr_sort(int64_t nv_total, const int32_t* __restrict__ off,
                           int32_t* __restrict__ ent) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv_total) return;
  const int32_t b = off[v], e = off[v + 1];
  for (int32_t i = b + 1; i < e; ++i) {
    const int32_t x = ent[i];
    int32_t j = i - 1;
    while (j >= b && ent[j] > x) {
      ent[j + 1] = ent[j];
      --j;
    }
    ent[j + 1] = x;
  }
}

// ---------------------------------------------------------------------------
// Host side: launch plans and launchers.

int num_sms() {
  static std::atomic<int> cached[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  int v = cached[dev].load();
  if (v <= 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    cached[dev].store(v);
  }
  return v;
}

static int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

namespace {
std::atomic<int> g_fwd_variant{0};
std::atomic<int> g_bwd_variant{0};
}  // namespace

int fwd_variant() { return g_fwd_variant.load(); }
int bwd_variant() { return g_bwd_variant.load(); }
void set_variants(int fwd, int bwd) {
  g_fwd_variant.store(fwd);
  g_bwd_variant.store(bwd);
}

void set_band_half(CellDesc& d, bool herm) {
  d.herm = herm ? 1 : 0;
  d.ne = herm ? (d.nband + 1) / 2 : d.nband;
}

void plan_cell_tiles(CellDesc& d) {
  plan_cell_tiles_for(d, kFwdVariants[fwd_variant()], kBwdVariants[bwd_variant()]);
}

void plan_cell_tiles_for(CellDesc& d, const FwdVariant& fv, const BwdVariant& bv) {
  const int64_t xtile = (int64_t)fv.NT * fv.R;
  d.xtiles = (int32_t)std::max<int64_t>(1, cdiv(d.ne, xtile));
  int64_t fsplit = std::max<int64_t>(1, cdiv((int64_t)num_sms() * fv.waves, d.xtiles));
  fsplit = std::min<int64_t>(fsplit, std::max<int64_t>(1, cdiv(d.nt, kFwdTF)));
  int64_t fchunk = cdiv(std::max<int64_t>(d.nt, 1), fsplit);
  fchunk = cdiv(fchunk, kFwdTF) * kFwdTF;
  d.fchunk = (int32_t)fchunk;
  d.fsplit = (int32_t)std::max<int64_t>(1, cdiv(d.nt, fchunk));

  const int64_t fblock = (int64_t)bv.NT * bv.F;
  d.fblocks = (int32_t)std::max<int64_t>(1, cdiv(d.nt, fblock));
  int64_t bch = std::max<int64_t>(1, cdiv((int64_t)num_sms() * bv.waves, d.fblocks));
  bch = std::min<int64_t>(bch, std::max<int64_t>(1, cdiv(d.ne, kBwdTX)));
  int64_t bx = cdiv(std::max<int64_t>(d.ne, 1), bch);
  bx = cdiv(bx, kBwdTX) * kBwdTX;
  d.bxchunk = (int32_t)bx;
  d.bchunks = (int32_t)std::max<int64_t>(1, cdiv(d.ne, bx));
}

void plan_offsets(CellDesc* cells, int ncells, PlanTotals& t) {
  t = PlanTotals{};
  t.fwd_var = fwd_variant();
  t.bwd_var = bwd_variant();
  for (int i = 0; i < ncells; ++i) {
    CellDesc& d = cells[i];
    plan_cell_tiles(d);
    d.v_off = t.nv;
    d.f_off = t.nt;
    d.b_off = t.nband;
    d.fpart_off = t.fpart;
    d.bpart_off = t.bpart;
    d.face_blk0 = (int32_t)t.face_blks;
    d.band_blk0 = (int32_t)t.band_blks;
    d.fwd_item0 = (int32_t)t.fwd_items;
    d.bwd_item0 = (int32_t)t.bwd_items;
    t.nv += d.nv;
    t.nt += d.nt;
    t.nband += d.nband;
    t.fpart += (int64_t)d.fsplit * d.ne;
    t.bpart += (int64_t)d.bchunks * 10 * d.nt;
    t.face_blks += std::max<int64_t>(1, cdiv(d.nt, kBlk));
    t.band_blks += std::max<int64_t>(1, cdiv(d.nband, kBlk));
    t.fwd_items += (int64_t)d.xtiles * d.fsplit;
    t.bwd_items += (int64_t)d.fblocks * d.bchunks;
  }
}

static int launch_status() {
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

int launch_face_prep(const Cells& c, const PlanTotals& t, const float* verts, const int64_t* faces,
                     const float* coeff, FaceRec* recs, double* area_part, int* err,
                     cudaStream_t st) {
  k_face_prep<<<(unsigned)t.face_blks, kBlk, 0, st>>>(c, verts, faces, coeff, recs, area_part, err);
  count_launches(1);
  return launch_status();
}

int launch_forward(const Cells& c, const PlanTotals& t, const FaceRec* recs,
                   const int32_t* band_index, const double* area_part, const float* otf,
                   float2* fpart, float2* ft_list, float2* grid, int* err, cudaStream_t st) {
  if (t.fwd_items > 0 && t.nband > 0) {
    profile_begin(0, st);
    const unsigned g = (unsigned)t.fwd_items;
    switch (t.fwd_var) {  // the variant the tiles were planned for
      case 1: k_meshft_fwd<2, 128, kFwdTF, kStages><<<g, 128, 0, st>>>(c, recs, nullptr, band_index, nullptr, fpart, err); break;
      case 2: k_meshft_fwd<4, 256, kFwdTF, kStages><<<g, 256, 0, st>>>(c, recs, nullptr, band_index, nullptr, fpart, err); break;
      case 3: k_meshft_fwd<8, 64, kFwdTF, kStages><<<g, 64, 0, st>>>(c, recs, nullptr, band_index, nullptr, fpart, err); break;
      case 4: k_meshft_fwd<4, 128, kFwdTF, kStages><<<g, 128, 0, st>>>(c, recs, nullptr, band_index, nullptr, fpart, err); break;
      case 5: k_meshft_fwd<2, 256, kFwdTF, kStages><<<g, 256, 0, st>>>(c, recs, nullptr, band_index, nullptr, fpart, err); break;
      default: k_meshft_fwd<4, 128, kFwdTF, kStages><<<g, 128, 0, st>>>(c, recs, nullptr, band_index, nullptr, fpart, err); break;
    }
    profile_end(0, st);
    count_launches(1);
    if (launch_status()) return DM_ERR_CUDA;
  }
  if (t.nband > 0) {
    k_meshft_fwd_epi<<<(unsigned)t.band_blks, kBlk, 0, st>>>(c, band_index, fpart, area_part, otf,
                                                            ft_list, grid, err);
    count_launches(1);
  }
  return launch_status();
}

int launch_backward(const Cells& c, const PlanTotals& t, const float* verts, const int64_t* faces,
                    const float* coeff, const FaceRec* recs, const double* area_part,
                    const int32_t* band_index, const float2* grad_list, const float2* grad_grid,
                    const float* otf, float grad_scale, const float2* ft_list, XiRec* xrec,
                    double* s_part, float* bpart, float* contrib, const int32_t* csr_off,
                    const int32_t* csr_ent, float* grad_verts, float* grad_coeff,
                    float* grad_otf_band, int32_t* key_hist, int32_t* key_first,
                    int32_t* face_order, int32_t* face_slot, int* err, cudaStream_t st) {
  // face order by size (see k_face_key_hist); skipped for small meshes
  const bool sort = face_order && t.nt >= kSortMinFaces;
  if (sort) {
    k_face_key_hist<<<(unsigned)t.face_blks, kBlk, 0, st>>>(c, recs, key_hist);
    k_face_key_scan<<<(unsigned)std::max(c.n, 1), kKeyBins, 0, st>>>(c, key_hist, key_first);
    k_face_key_scatter<<<(unsigned)t.face_blks, kBlk, 0, st>>>(c, recs, key_first, face_order,
                                                               face_slot);
    count_launches(3);
    if (launch_status()) return DM_ERR_CUDA;
  }
  const int32_t* order = sort ? face_order : nullptr;
  const int32_t* slot_of = sort ? face_slot : nullptr;
  k_bwd_band_prep<<<(unsigned)t.band_blks, kBlk, 0, st>>>(c, band_index, grad_list, grad_grid, otf,
                                                         grad_scale, ft_list, xrec, grad_otf_band,
                                                         s_part, err);
  count_launches(1);
  if (launch_status()) return DM_ERR_CUDA;
  if (t.bwd_items > 0 && t.nband > 0 && t.nt > 0) {
    cudaMemsetAsync(bpart, 0, sizeof(float) * (size_t)std::max<int64_t>(t.bpart, 1), st);
    profile_begin(1, st);
    const unsigned g = (unsigned)t.bwd_items;
    switch (t.bwd_var) {  // the variant the tiles were planned for
      case 1: k_meshft_bwd<1, 128, kBwdTX, kStages><<<g, 128, 0, st>>>(c, recs, nullptr, xrec, nullptr, order, bpart, err); break;
      case 2: k_meshft_bwd<2, 64, kBwdTX, kStages><<<g, 64, 0, st>>>(c, recs, nullptr, xrec, nullptr, order, bpart, err); break;
      case 3: k_meshft_bwd<1, 256, kBwdTX, kStages><<<g, 256, 0, st>>>(c, recs, nullptr, xrec, nullptr, order, bpart, err); break;
      case 4: k_meshft_bwd<2, 128, kBwdTX, kStages><<<g, 128, 0, st>>>(c, recs, nullptr, xrec, nullptr, order, bpart, err); break;
      case 5: k_meshft_bwd<1, 128, kBwdTX, kStages><<<g, 128, 0, st>>>(c, recs, nullptr, xrec, nullptr, order, bpart, err); break;
      case 6: k_meshft_bwd<2, 128, kBwdTX, kStages, false, XiRec, 5><<<g, 128, 0, st>>>(c, recs, nullptr, xrec, nullptr, order, bpart, err); break;
      case 7: k_meshft_bwd<2, 128, kBwdTX, kStages, false, XiRec, 6><<<g, 128, 0, st>>>(c, recs, nullptr, xrec, nullptr, order, bpart, err); break;
      case 8: k_meshft_bwd<1, 128, kBwdTX, kStages, false, XiRec, 8><<<g, 128, 0, st>>>(c, recs, nullptr, xrec, nullptr, order, bpart, err); break;
      default: k_meshft_bwd<2, 128, kBwdTX, kStages><<<g, 128, 0, st>>>(c, recs, nullptr, xrec, nullptr, order, bpart, err); break;
    }
    profile_end(1, st);
    count_launches(1);
    if (launch_status()) return DM_ERR_CUDA;
  } else if (t.bpart > 0) {
    cudaMemsetAsync(bpart, 0, sizeof(float) * (size_t)t.bpart, st);
  }
  k_bwd_face_epi<<<(unsigned)t.face_blks, kBlk, 0, st>>>(c, verts, faces, coeff, area_part, s_part,
                                                        bpart, slot_of, contrib, grad_coeff);
  count_launches(1);
  if (launch_status()) return DM_ERR_CUDA;
  if (t.nv > 0) {
    k_vertex_gather<<<(unsigned)cdiv(t.nv, kBlk), kBlk, 0, st>>>(t.nv, csr_off, csr_ent, contrib,
                                                                grad_verts);
    count_launches(1);
  }
  return launch_status();
}

int launch_vertex_gather(int64_t nv, const int32_t* csr_off, const int32_t* csr_ent,
                         const float* contrib, float* grad_verts, cudaStream_t st) {
  if (nv > 0) {
    k_vertex_gather<<<(unsigned)cdiv(nv, kBlk), kBlk, 0, st>>>(nv, csr_off, csr_ent, contrib,
                                                              grad_verts);
    count_launches(1);
  }
  return launch_status();
}

int launch_topology(const Cells& c, const PlanTotals& t, const int64_t* faces, int32_t* count,
                    int32_t* off, int32_t* cursor, int32_t* ent, int* err, cudaStream_t st) {
  cudaMemsetAsync(count, 0, sizeof(int32_t) * (size_t)(t.nv + 1), st);
  cudaMemsetAsync(cursor, 0, sizeof(int32_t) * (size_t)(t.nv + 1), st);
  if (t.nt > 0) k_csr_count<<<(unsigned)t.face_blks, kBlk, 0, st>>>(c, faces, count, err);
  k_csr_scan<<<1, 1024, 0, st>>>(count, off, t.nv);
  if (t.nt > 0) k_csr_fill<<<(unsigned)t.face_blks, kBlk, 0, st>>>(c, faces, off, cursor, ent);
  if (t.nv > 0) k_csr_sort<<<(unsigned)cdiv(t.nv, kBlk), kBlk, 0, st>>>(t.nv, off, ent);
  count_launches(2 + (t.nt > 0 ? 2 : 0) + (t.nv > 0 ? 1 : 0));
  return launch_status();
}

// ---------------------------------------------------------------------------
// Explicit frequency lists (forward_fourier3d_cpp / backward_fourier3d_cpp,
// fourier3d_cuda.cpp:27-65): frequencies off any grid, vertex coordinates as
// given.  The cell has lower corner 0 and per-axis length L_d = 2.5 max|v_d|
// (computed on the device, so |v_d| < L_d / 2 and the fixed-point positions fit
// in int32); each frequency becomes m_d = xi_d L_d / pi, split into its nearest
// integer and a remainder (split phase, pair_math.cuh).  The same main kernels
// run with the off-grid records; every frequency is evaluated.

constexpr FwdVariant kXiFwd{2, 256, 16};
constexpr BwdVariant kXiBwd{1, 128, 16};

// One block: L_d from the vertices, written with the host plan into *out.
__global__ void k_xi_cell(CellDesc base, const float* __restrict__ verts, int64_t nv,
                          CellDesc* __restrict__ out, int* err) {
  __shared__ float sh[3][32];
  float m[3] = {0.f, 0.f, 0.f};
  bool fin = true;
  for (int64_t i = threadIdx.x; i < nv; i += blockDim.x)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float a = fabsf(verts[3 * i + j]);
      if (isfinite(a)) m[j] = fmaxf(m[j], a); else fin = false;
    }
  if (!fin) set_error(err, DM_ERR_NONFINITE);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    for (int o = 16; o > 0; o >>= 1) m[j] = fmaxf(m[j], __shfl_down_sync(0xffffffffu, m[j], o));
    if ((threadIdx.x & 31) == 0) sh[j][threadIdx.x >> 5] = m[j];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    CellDesc d = base;
    for (int j = 0; j < 3; ++j) {
      float v = 0.f;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v = fmaxf(v, sh[j][w]);
      d.lo[j] = 0.0;
      d.len[j] = v > 0.f ? 2.5 * (double)v : 1.0;
    }
    *out = d;
  }
}

// Off-grid frequency records (and, with a cotangent, g and per-block sums of
// s = Re(conj(g) ft)).
__global__ void k_xi_prep(const CellDesc* __restrict__ dp, const float* __restrict__ xi_list,
                          const float2* __restrict__ grad_list, float grad_scale,
                          const float2* __restrict__ ft_list, XiRecOff* __restrict__ xr,
                          double* __restrict__ s_part, int* err) {
  __shared__ double sh[40];
  const CellDesc d = *dp;
  const int m = blockIdx.x * kBlk + threadIdx.x;
  double s = 0.0;
  if (m < d.nband) {
    XiRecOff r;
    bool ok = true;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double mm = (double)xi_list[3 * (int64_t)m + j] * d.len[j] * 0.3183098861837907;
      if (!(fabs(mm) < 1073741824.0)) {  // |m| < 2^30 (NaN fails too)
        ok = false;
        r.mi[j] = 0;
        r.mf[j] = 0.f;
        r.fr[j] = 0.f;
        continue;
      }
      const double mi = rint(mm);
      r.mi[j] = (int32_t)mi;
      r.mf[j] = (float)mm;
      r.fr[j] = (float)(mm - mi);
    }
    if (!ok) set_error(err, DM_ERR_SIZE);
    r.g_re = r.g_im = r.pad = 0.f;
    if (grad_list) {
      const float2 g = grad_list[m];
      r.g_re = grad_scale * g.x;
      r.g_im = grad_scale * g.y;
      const float2 ft = ft_list[m];
      s = (double)r.g_re * ft.x + (double)r.g_im * ft.y;
    }
    xr[m] = r;
  }
  if (s_part) {
    const double t = block_sum_d(s, sh);
    if (threadIdx.x == 0) s_part[blockIdx.x] = t;
  }
}

// ft_list = (2/M) sum over splits, fixed order.
__global__ void k_xi_fwd_epi(const CellDesc* __restrict__ dp, const float2* __restrict__ fpart,
                             const double* __restrict__ area_part, int n_area,
                             float2* __restrict__ ft_list) {
  __shared__ double sh[40];
  const CellDesc d = *dp;
  const double M = block_sum_list(area_part, n_area, sh);
  const int m = blockIdx.x * kBlk + threadIdx.x;
  if (m >= d.nband) return;
  double sx = 0.0, sy = 0.0;
  for (int s = 0; s < d.fsplit; ++s) {
    const float2 v = fpart[(int64_t)s * d.nband + m];
    sx += v.x;
    sy += v.y;
  }
  const double sc = d.nt > 0 ? 2.0 / M : 0.0;
  ft_list[m] = make_float2((float)(sx * sc), (float)(sy * sc));
}

CellDesc plan_xi_cell(int64_t nv, int64_t nt, int64_t n_xi, PlanTotals& t) {
  CellDesc d;
  memset(&d, 0, sizeof(d));
  for (int k = 0; k < 3; ++k) {
    d.len[k] = 1.0;
    d.n[k] = 1;
  }
  d.nv = (int32_t)nv;
  d.nt = (int32_t)nt;
  d.nband = (int32_t)n_xi;
  set_band_half(d, false);
  plan_cell_tiles_for(d, kXiFwd, kXiBwd);
  t = PlanTotals{};
  t.nv = nv;
  t.nt = nt;
  t.nband = n_xi;
  t.fpart = (int64_t)d.fsplit * d.ne;
  t.bpart = (int64_t)d.bchunks * 10 * d.nt;
  t.face_blks = std::max<int64_t>(1, cdiv(nt, kBlk));
  t.band_blks = std::max<int64_t>(1, cdiv(n_xi, kBlk));
  t.fwd_items = (int64_t)d.xtiles * d.fsplit;
  t.bwd_items = (int64_t)d.fblocks * d.bchunks;
  return d;
}

int launch_xi_forward(const CellDesc& plan, const PlanTotals& t, const float* verts,
                      const int64_t* faces, const float* coeff, const float* xi_list,
                      CellDesc* dev_desc, FaceRec* recs, double* area_part, XiRecOff* xr,
                      float2* fpart, float2* ft_list, int* err, cudaStream_t st) {
  k_xi_cell<<<1, 1024, 0, st>>>(plan, verts, t.nv, dev_desc, err);
  Cells c;
  memset(&c, 0, sizeof(c));
  c.p = dev_desc;
  c.n = 1;
  count_launches(1);
  if (t.nt > 0) {
    k_face_prep<<<(unsigned)t.face_blks, kBlk, 0, st>>>(c, verts, faces, coeff, recs, area_part,
                                                       err);
    count_launches(1);
  }
  if (t.nband <= 0) return launch_status();
  k_xi_prep<<<(unsigned)t.band_blks, kBlk, 0, st>>>(dev_desc, xi_list, nullptr, 0.f, nullptr,
                                                   xr, nullptr, err);
  count_launches(1);
  if (t.nt > 0) {
    k_meshft_fwd<kXiFwd.R, kXiFwd.NT, kFwdTF, kStages, false, true>
        <<<(unsigned)t.fwd_items, kXiFwd.NT, 0, st>>>(c, recs, nullptr, nullptr, xr, fpart, err);
    count_launches(1);
  } else {
    cudaMemsetAsync(fpart, 0, sizeof(float2) * (size_t)std::max<int64_t>(t.fpart, 1), st);
    cudaMemsetAsync(area_part, 0, sizeof(double), st);
  }
  k_xi_fwd_epi<<<(unsigned)t.band_blks, kBlk, 0, st>>>(dev_desc, fpart, area_part,
                                                      (int)(t.nt > 0 ? t.face_blks : 1), ft_list);
  count_launches(1);
  return launch_status();
}

int launch_xi_backward(const CellDesc& plan, const PlanTotals& t, const float* verts,
                       const int64_t* faces, const float* coeff, const float* xi_list,
                       const float2* grad_list, float grad_scale, const float2* ft_list,
                       const int32_t* csr_off, const int32_t* csr_ent, CellDesc* dev_desc,
                       FaceRec* recs, double* area_part, XiRecOff* xr, double* s_part,
                       float* bpart, float* contrib, float* grad_verts, float* grad_coeff,
                       int32_t* key_hist, int32_t* key_first, int32_t* face_order,
                       int32_t* face_slot, int* err, cudaStream_t st) {
  if (t.nt <= 0) {
    if (t.nv > 0) cudaMemsetAsync(grad_verts, 0, sizeof(float) * 3 * (size_t)t.nv, st);
    return launch_status();
  }
  k_xi_cell<<<1, 1024, 0, st>>>(plan, verts, t.nv, dev_desc, err);
  Cells c;
  memset(&c, 0, sizeof(c));
  c.p = dev_desc;
  c.n = 1;
  k_face_prep<<<(unsigned)t.face_blks, kBlk, 0, st>>>(c, verts, faces, coeff, recs, area_part,
                                                     err);
  count_launches(2);
  const bool sort = t.nt >= kSortMinFaces;
  if (sort) {
    k_face_key_hist<<<(unsigned)t.face_blks, kBlk, 0, st>>>(c, recs, key_hist);
    k_face_key_scan<<<1, kKeyBins, 0, st>>>(c, key_hist, key_first);
    k_face_key_scatter<<<(unsigned)t.face_blks, kBlk, 0, st>>>(c, recs, key_first, face_order,
                                                               face_slot);
    count_launches(3);
  }
  if (t.nband > 0) {
    k_xi_prep<<<(unsigned)t.band_blks, kBlk, 0, st>>>(dev_desc, xi_list, grad_list, grad_scale,
                                                     ft_list, xr, s_part, err);
    cudaMemsetAsync(bpart, 0, sizeof(float) * (size_t)std::max<int64_t>(t.bpart, 1), st);
    k_meshft_bwd<kXiBwd.F, kXiBwd.NT, kBwdTX, kStages, false, XiRecOff>
        <<<(unsigned)t.bwd_items, kXiBwd.NT, 0, st>>>(c, recs, nullptr, xr, nullptr,
                                                      sort ? face_order : nullptr, bpart, err);
    count_launches(2);
  } else {
    cudaMemsetAsync(s_part, 0, sizeof(double), st);
    cudaMemsetAsync(bpart, 0, sizeof(float) * (size_t)std::max<int64_t>(t.bpart, 1), st);
  }
  k_bwd_face_epi<<<(unsigned)t.face_blks, kBlk, 0, st>>>(c, verts, faces, coeff, area_part,
                                                        s_part, bpart,
                                                        sort ? face_slot : nullptr, contrib,
                                                        grad_coeff);
  count_launches(1);
  return launch_vertex_gather(t.nv, csr_off, csr_ent, contrib, grad_verts, st);
}

}  // namespace dm
