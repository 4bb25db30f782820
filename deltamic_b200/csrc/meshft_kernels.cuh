// Main meshFT kernels and the device helpers they share; included by meshft.cu
// (the surface transform of Fourier3dMesh) and volume.cu (surface plus
// enclosed-volume transform of the autofluorescence variant).
//
//  * forward: item = (cell, frequency tile of NT*R, face split).  Each thread
//    owns R band frequencies and loops over the faces of its split; face records
//    are staged in shared memory by the bulk-copy engine in a ring of NS tiles
//    and read as broadcasts.  Partial sums per (split, frequency) go to HBM and
//    the epilogue adds them in a fixed order -> deterministic, no atomics.
//  * backward: item = (cell, face block of NT*F, frequency chunk).  Each thread
//    owns F faces (geometry and its accumulators in registers) and loops over the
//    frequencies of its chunk, staged in shared memory the same way.  Per-face
//    partials go to HBM; a face epilogue reduces chunks in a fixed order.
//
// With kVol the per-pair weight is complex and frequency dependent,
//   W_k(xi) = a_k + i beta (xi . nor_k) / |xi|^2
// (render.py:228-318): the forward keeps a second accumulator sum_k F_k (xi.nor_k)
// per frequency (written as a second block of partials), and the adjoint takes a
// per-face weight record {a_k, beta nor'_k} and a per-frequency record of
// g / |xi|^2 next to the cotangent.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "dm_common.cuh"
#include "pair_math.cuh"

namespace dm {

constexpr int kBlk = 256;  // threads of the element-wise kernels

// ---------------------------------------------------------------------------
// helpers

__device__ __forceinline__ void band_to_m(int32_t idx, const CellDesc& d, int32_t mi[3]) {
  const int32_t n12 = d.n[1] * d.n[2];
  const int32_t k0 = idx / n12;
  const int32_t rem = idx - k0 * n12;
  const int32_t k1 = rem / d.n[2];
  const int32_t k2 = rem - k1 * d.n[2];
  mi[0] = 2 * k0 - (d.n[0] - 1);
  mi[1] = 2 * k1 - (d.n[1] - 1);
  mi[2] = 2 * k2 - (d.n[2] - 1);
}

__device__ __forceinline__ FaceGeom geom_from_rec(const FaceRec& r) {
  FaceGeom g;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    g.Ua[d] = r.Ua[d];
    g.Ub[d] = r.Ub[d];
    g.Uc[d] = r.Uc[d];
    g.hab[d] = r.hab[d];
    g.hbc[d] = r.hbc[d];
  }
  return g;
}

__device__ __forceinline__ void load_rec_shared(const FaceRec* p, FaceRec& r) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  uint4* o = reinterpret_cast<uint4*>(&r);
  o[0] = q[0];
  o[1] = q[1];
  o[2] = q[2];
  o[3] = q[3];
}

// Block-wide sum in double (fixed order), result valid in thread 0.
__device__ __forceinline__ double block_sum_d(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    for (int i = 0; i < nw; ++i) r += sh[i];
  }
  __syncthreads();
  return r;
}

// Sum of ``n`` doubles (fixed order), broadcast to the whole block.
__device__ __forceinline__ double block_sum_list(const double* p, int n, double* sh) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += p[i];
  double r = block_sum_d(v, sh);
  if (threadIdx.x == 0) sh[32] = r;
  __syncthreads();
  r = sh[32];
  __syncthreads();
  return r;
}

// Cotangent of band entry gm (0 for an invalid voxel index).
__device__ __forceinline__ float2 band_cotangent(const CellDesc& d, int64_t gm, int32_t idx,
                                                 bool ok, const float2* __restrict__ grad_list,
                                                 const float2* __restrict__ grad_grid,
                                                 const float* __restrict__ otf,
                                                 float grad_scale, float2& G) {
  if (!ok) {
    G = make_float2(0.f, 0.f);
    return G;
  }
  G = grad_list ? grad_list[gm] : grad_grid[d.grid_off + idx];
  const float gs = grad_scale * (otf ? otf[d.grid_off + idx] : 1.0f);
  return make_float2(gs * G.x, gs * G.y);
}

// One bulk copy of ``cnt`` records from src + first into dst and, with kExtra, of
// the matching float4 records of ``extra`` into xdst, completing on one barrier.
template <bool kExtra, typename Rec>
__device__ __forceinline__ void stage_tile(Rec* dst, float4* xdst, const Rec* src,
                                           const float4* extra, int first, int cnt,
                                           uint64_t* bar) {
  const uint32_t b0 = (uint32_t)cnt * (uint32_t)sizeof(Rec);
  const uint32_t b1 = kExtra ? (uint32_t)cnt * (uint32_t)sizeof(float4) : 0u;
  mbar_expect_tx(bar, b0 + b1);
  bulk_g2s(dst, src + first, b0, bar);
  if (kExtra) bulk_g2s(xdst, extra + first, b1, bar);
}

// ---------------------------------------------------------------------------
// Forward main kernel.

// acc += ac F and, with kVol, vac += (m . nv) F for every frequency of the thread.
template <int R, bool kVol, class XV>
__device__ __forceinline__ void fwd_face(const FaceGeom& g, float ac, const float4& nv,
                                         const XV (&xv)[R], float2 (&acc)[R],
                                         float2 (&vac)[R]) {
  uint32_t spm = 0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    c32 F;
    if (pair_forward(xv[r], g, F)) {
      acc[r].x += ac * F.x;
      acc[r].y += ac * F.y;
      if (kVol) {
        const float t = xv[r].mf[0] * nv.x + xv[r].mf[1] * nv.y + xv[r].mf[2] * nv.z;
        vac[r].x += t * F.x;
        vac[r].y += t * F.y;
      }
    } else {
      spm |= 1u << r;
    }
  }
  if (spm) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if ((spm >> r) & 1u) {
        const c32 F = pair_forward_degenerate(xv[r], g);
        acc[r].x += ac * F.x;
        acc[r].y += ac * F.y;
        if (kVol) {
          const float t = xv[r].mf[0] * nv.x + xv[r].mf[1] * nv.y + xv[r].mf[2] * nv.z;
          vac[r].x += t * F.x;
          vac[r].y += t * F.y;
        }
      }
    }
  }
}

// Two frequencies of one thread against one face with paired FP32 on the series
// path (both pairs series with one coefficient set), scalar otherwise; lane x/y
// of accx/accy accumulates frequency 0/1.  mf2[d] = {mf_d(xi0), mf_d(xi1)}.
template <class XV>
__device__ __forceinline__ void fwd_face2(const FaceGeom& g, float ac, const XV (&xv)[2],
                                          const v2 (&mf2)[3], v2& accx, v2& accy) {
  const v2 hab = fma2(mf2[0], B2(g.hab[0]), fma2(mf2[1], B2(g.hab[1]), mul2(mf2[2], B2(g.hab[2]))));
  const v2 hbc = fma2(mf2[0], B2(g.hbc[0]), fma2(mf2[1], B2(g.hbc[1]), mul2(mf2[2], B2(g.hbc[2]))));
  const v2 hca = neg2(add2(hab, hbc));
  if (series_pair2(hab, hbc, hca)) {
    v2 Fx, Fy;
    if (series_short2(hab, hbc, hca))
      forward_series2<true>(xv[0], xv[1], g.Ua, hab, hca, Fx, Fy);
    else
      forward_series2<false>(xv[0], xv[1], g.Ua, hab, hca, Fx, Fy);
    accx = fma2(B2(ac), Fx, accx);
    accy = fma2(B2(ac), Fy, accy);
    return;
  }
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    c32 F;
    if (!pair_forward(xv[r], g, F)) F = pair_forward_degenerate(xv[r], g);
    if (r == 0) {
      accx.x += ac * F.x;
      accy.x += ac * F.y;
    } else {
      accx.y += ac * F.x;
      accy.y += ac * F.y;
    }
  }
}

// Frequency of an XiRecOff (off-grid xi list).
__device__ __forceinline__ XiValOff xi_off(const XiRecOff& r) {
  XiValOff x;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    x.mi[k] = r.mi[k];
    x.mf[k] = r.mf[k];
    x.fr[k] = r.fr[k];
  }
  return x;
}

// fpart[split][m] = sum over the split's faces of area_coeff F; with kVol also
// fpart[fsplit + split][m] = sum of (m . nor') F, nor' = vrec[f].xyz.  With kOff
// the frequencies are the off-grid records xoff (split phase), else band voxels.
template <int R, int NT, int TF, int NS, bool kVol = false, bool kOff = false>
__global__ void __launch_bounds__(NT) k_meshft_fwd(Cells cells, const FaceRec* __restrict__ recs,
                                                  const float4* __restrict__ vrec,
                                                  const int32_t* __restrict__ band_index,
                                                  const XiRecOff* __restrict__ xoff,
                                                  float2* __restrict__ fpart, int* err) {
  using XV = typename std::conditional<kOff, XiValOff, XiVal>::type;
  __shared__ __align__(128) FaceRec sf[NS][TF];
  __shared__ __align__(16) float4 sv[kVol ? NS : 1][kVol ? TF : 1];
  __shared__ __align__(8) uint64_t bar[NS];
  const int item = blockIdx.x;
  const int ci = cell_find(cells, item, [](const CellDesc& d) { return d.fwd_item0; });
  const CellDesc d = cell_get(cells, ci);
  const int local = item - d.fwd_item0;
  const int xt = local % d.xtiles;
  const int split = local / d.xtiles;
  const int f0 = split * d.fchunk;
  const int nf = min(d.nt, f0 + d.fchunk) - f0;
  if (d.ne <= 0) return;
  if (nf <= 0) {  // no faces: the partial sums are zero
    for (int r = 0; r < R; ++r) {
      const int m = xt * NT * R + r * NT + threadIdx.x;
      if (m < d.ne) {
        fpart[d.fpart_off + (int64_t)split * d.ne + m] = make_float2(0.f, 0.f);
        if (kVol) fpart[d.fpart_off + (int64_t)(d.fsplit + split) * d.ne + m] = make_float2(0.f, 0.f);
      }
    }
    return;
  }

  XV xv[R];
  int mloc[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int m = xt * NT * R + r * NT + threadIdx.x;
    mloc[r] = m;
    // lanes past the band evaluate a real frequency so every lane takes the
    // same branches; their sums are never stored
    const int mm = min(m, d.ne - 1);
    if constexpr (kOff) {
      xv[r] = xi_off(xoff[d.b_off + mm]);
    } else {
      band_to_m(band_index[d.b_off + mm], d, xv[r].mi);
#pragma unroll
      for (int k = 0; k < 3; ++k) xv[r].mf[k] = (float)xv[r].mi[k];
    }
  }

  const int ntiles = (nf + TF - 1) / TF;
  const FaceRec* src0 = recs + d.f_off + f0;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int s = 0; s < NS && s < ntiles; ++s)
      stage_tile<kVol>(&sf[s][0], &sv[kVol ? s : 0][0], src0, vrec + d.f_off + f0, s * TF,
                       min(TF, nf - s * TF), &bar[s]);
  }

  float2 acc[R], vac[R];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r] = vac[r] = make_float2(0.f, 0.f);

  for (int t = 0; t < ntiles; ++t) {
    const int s = t % NS;
    if (!mbar_wait_bounded(&bar[s], (uint32_t)((t / NS) & 1), err)) return;
    const int nft = min(TF, nf - t * TF);
    float2 tacc[R], tvac[R];
#pragma unroll
    for (int r = 0; r < R; ++r) tacc[r] = tvac[r] = make_float2(0.f, 0.f);
    if constexpr (R == 2 && !kVol) {
      // paired FP32: both frequencies of the thread per face
      v2 mf2[3], ax = B2(0.f), ay = B2(0.f);
#pragma unroll
      for (int k = 0; k < 3; ++k) mf2[k] = v2{xv[0].mf[k], xv[1].mf[k]};
      for (int j = 0; j < nft; ++j) {
        FaceRec fr;
        load_rec_shared(&sf[s][j], fr);
        fwd_face2(geom_from_rec(fr), fr.area_coeff, xv, mf2, ax, ay);
      }
      tacc[0] = make_float2(ax.x, ay.x);
      tacc[1] = make_float2(ax.y, ay.y);
    } else {
      for (int j = 0; j < nft; ++j) {
        FaceRec fr;
        load_rec_shared(&sf[s][j], fr);
        const float4 nv = kVol ? sv[s][j] : make_float4(0.f, 0.f, 0.f, 0.f);
        fwd_face<R, kVol>(geom_from_rec(fr), fr.area_coeff, nv, xv, tacc, tvac);
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      acc[r].x += tacc[r].x;
      acc[r].y += tacc[r].y;
      if (kVol) {
        vac[r].x += tvac[r].x;
        vac[r].y += tvac[r].y;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && t + NS < ntiles) {
      fence_proxy_async();
      const int tn = t + NS;
      stage_tile<kVol>(&sf[s][0], &sv[kVol ? s : 0][0], src0, vrec + d.f_off + f0, tn * TF,
                       min(TF, nf - tn * TF), &bar[s]);
    }
  }
  float2* out = fpart + d.fpart_off + (int64_t)split * d.ne;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (mloc[r] < d.ne) {
      out[mloc[r]] = acc[r];
      if (kVol) out[(int64_t)d.fsplit * d.ne + mloc[r]] = vac[r];
    }
  }
}

// ---------------------------------------------------------------------------
// Backward main kernel.
//
// Accumulators per face: q[3v+j] = sum z_v m_j (v = a,b,c), q[9] = sum Re(conj(g) F)
// and, with kVol, q[10+j] = sum Re(i conj(g/|xi|^2) F) m_j.
template <bool kVol>
struct BwdAccT {
  static constexpr int N = kVol ? 13 : 10;
  float q[N];
};

template <bool kVol>
__device__ __forceinline__ void bwd_accumulate(BwdAccT<kVol>& a, const float z[3], float r,
                                               const float mf[3], float s) {
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    a.q[3 * v + 0] += z[v] * mf[0];
    a.q[3 * v + 1] += z[v] * mf[1];
    a.q[3 * v + 2] += z[v] * mf[2];
  }
  a.q[9] += r;
  if constexpr (kVol) {
    a.q[10] += s * mf[0];
    a.q[11] += s * mf[1];
    a.q[12] += s * mf[2];
  }
}

// bpart[chunk][i][f] = q[i] of face slot f over the chunk's frequencies.  With
// kVol, fw[face] = {a, beta nor'} and xg[m] = {Re, Im} of g / |xi|^2 (0 at xi = 0);
// the pair's cotangent for z is g conj(W) = a g - i (beta m.nor') g/|xi|^2.
// Frequency and cotangent of a staged record (grid or off-grid).
__device__ __forceinline__ void load_xi(const XiRec& r, XiVal& xv, float& gre, float& gim) {
  const uint4* q = reinterpret_cast<const uint4*>(&r);
  const uint4 w0 = q[0], w1 = q[1];
  xv.mi[0] = (int32_t)w0.x;
  xv.mi[1] = (int32_t)w0.y;
  xv.mi[2] = (int32_t)w0.z;
  gre = __uint_as_float(w0.w);
  xv.mf[0] = __uint_as_float(w1.x);
  xv.mf[1] = __uint_as_float(w1.y);
  xv.mf[2] = __uint_as_float(w1.z);
  gim = __uint_as_float(w1.w);
}
__device__ __forceinline__ void load_xi(const XiRecOff& r, XiValOff& xv, float& gre,
                                        float& gim) {
  const uint4* q = reinterpret_cast<const uint4*>(&r);
  const uint4 w0 = q[0], w1 = q[1], w2 = q[2];
  xv.mi[0] = (int32_t)w0.x;
  xv.mi[1] = (int32_t)w0.y;
  xv.mi[2] = (int32_t)w0.z;
  gre = __uint_as_float(w0.w);
  xv.mf[0] = __uint_as_float(w1.x);
  xv.mf[1] = __uint_as_float(w1.y);
  xv.mf[2] = __uint_as_float(w1.z);
  gim = __uint_as_float(w1.w);
  xv.fr[0] = __uint_as_float(w2.x);
  xv.fr[1] = __uint_as_float(w2.y);
  xv.fr[2] = __uint_as_float(w2.z);
}

// MINB > 0 caps the registers for MINB CTAs per SM; 0 leaves the choice to ptxas.
template <int F, int NT, int TX, int NS, bool kVol = false, class XR = XiRec, int MINB = 0>
__global__ void __launch_bounds__(NT, MINB) k_meshft_bwd(Cells cells, const FaceRec* __restrict__ recs,
                                                  const float4* __restrict__ fw,
                                                  const XR* __restrict__ xrec,
                                                  const float4* __restrict__ xg,
                                                  const int32_t* __restrict__ order,
                                                  float* __restrict__ bpart, int* err) {
  using Acc = BwdAccT<kVol>;
  using XV = typename std::conditional<std::is_same<XR, XiRecOff>::value, XiValOff, XiVal>::type;
  constexpr int NQ = Acc::N;
  __shared__ __align__(128) XR sx[NS][TX];
  __shared__ __align__(16) float4 sg[kVol ? NS : 1][kVol ? TX : 1];
  __shared__ __align__(8) uint64_t bar[NS];
  const int item = blockIdx.x;
  const int ci = cell_find(cells, item, [](const CellDesc& d) { return d.bwd_item0; });
  const CellDesc d = cell_get(cells, ci);
  const int local = item - d.bwd_item0;
  const int fb = local % d.fblocks;
  const int chunk = local / d.fblocks;
  const int x0 = chunk * d.bxchunk;
  const int nx = min(d.ne, x0 + d.bxchunk) - x0;
  if (nx <= 0 || d.nt <= 0) return;

  FaceGeom geom[F];
  float4 wt[F];
  int fidx[F];
#pragma unroll
  for (int k = 0; k < F; ++k) {
    const int f = fb * NT * F + k * NT + threadIdx.x;
    fidx[k] = f;
    // lanes past the last face evaluate a real face (never stored); with a face
    // order, slot f holds face order[f] (faces of similar size share a warp)
    const int64_t slot = d.f_off + min(f, d.nt - 1);
    const int64_t gf = order ? (int64_t)order[slot] : slot;
    geom[k] = geom_from_rec(recs[gf]);
    wt[k] = kVol ? fw[gf] : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  // edge vectors of the thread's first and last face as lane pairs (paired FP32)
  v2 hab2[3], hbc2[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    hab2[c] = v2{geom[0].hab[c], geom[F - 1].hab[c]};
    hbc2[c] = v2{geom[0].hbc[c], geom[F - 1].hbc[c]};
  }

  const int ntiles = (nx + TX - 1) / TX;
  const XR* src0 = xrec + d.b_off + x0;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int s = 0; s < NS && s < ntiles; ++s)
      stage_tile<kVol>(&sx[s][0], &sg[kVol ? s : 0][0], src0, xg + d.b_off + x0, s * TX,
                       min(TX, nx - s * TX), &bar[s]);
  }

  Acc acc[F];
#pragma unroll
  for (int k = 0; k < F; ++k)
#pragma unroll
    for (int i = 0; i < NQ; ++i) acc[k].q[i] = 0.f;

  for (int t = 0; t < ntiles; ++t) {
    const int s = t % NS;
    if (!mbar_wait_bounded(&bar[s], (uint32_t)((t / NS) & 1), err)) return;
    const int nxt = min(TX, nx - t * TX);
    Acc tacc[F];
#pragma unroll
    for (int k = 0; k < F; ++k)
#pragma unroll
      for (int i = 0; i < NQ; ++i) tacc[k].q[i] = 0.f;
    if constexpr (F == 2 && !kVol) {
      // paired FP32: both faces of the thread per frequency; lane x/y = face 0/1
      v2 q2[10];
#pragma unroll
      for (int i = 0; i < 10; ++i) q2[i] = B2(0.f);
      auto accum2 = [&](const v2 (&z)[3], v2 r, v2 m0, v2 m1, v2 m2) {
#pragma unroll
        for (int v = 0; v < 3; ++v) {
          q2[3 * v + 0] = fma2(z[v], m0, q2[3 * v + 0]);
          q2[3 * v + 1] = fma2(z[v], m1, q2[3 * v + 1]);
          q2[3 * v + 2] = fma2(z[v], m2, q2[3 * v + 2]);
        }
        q2[9] = add2(q2[9], r);
      };
      // one frequency: packed when both faces take the series path, else per face
      auto one = [&](int j) {
        XV xv;
        float gre, gim;
        load_xi(sx[s][j], xv, gre, gim);
        const v2 m0 = B2(xv.mf[0]), m1 = B2(xv.mf[1]), m2 = B2(xv.mf[2]);
        const v2 hab = fma2(m0, hab2[0], fma2(m1, hab2[1], mul2(m2, hab2[2])));
        const v2 hbc = fma2(m0, hbc2[0], fma2(m1, hbc2[1], mul2(m2, hbc2[2])));
        const v2 hca = neg2(add2(hab, hbc));
        if (series_pair2(hab, hbc, hca)) {
          v2 z[3], r;
          if (series_short2(hab, hbc, hca))
            adjoint_series2<true>(xv, geom[0].Ua, geom[1].Ua, hab, hca, gre, gim, z, r);
          else
            adjoint_series2<false>(xv, geom[0].Ua, geom[1].Ua, hab, hca, gre, gim, z, r);
          accum2(z, r, m0, m1, m2);
          return;
        }
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          float z[3], r;
          if (!pair_adjoint(xv, geom[k], gre, gim, z, r))
            pair_adjoint_degenerate(xv, geom[k], gre, gim, z, r);
#pragma unroll
          for (int v = 0; v < 3; ++v)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              float& a = k == 0 ? q2[3 * v + c].x : q2[3 * v + c].y;
              a += z[v] * xv.mf[c];
            }
          float& a9 = k == 0 ? q2[9].x : q2[9].y;
          a9 += r;
        }
      };
      for (int j = 0; j < nxt; ++j) one(j);
#pragma unroll
      for (int i = 0; i < 10; ++i) {
        tacc[0].q[i] = q2[i].x;
        tacc[F - 1].q[i] = q2[i].y;
      }
    } else {
      for (int j = 0; j < nxt; ++j) {
        XV xv;
        float gre, gim;
        load_xi(sx[s][j], xv, gre, gim);
        float2 gv = make_float2(0.f, 0.f);
        if (kVol) {
          const float4 g4 = sg[s][j];
          gv = make_float2(g4.x, g4.y);
        }
        uint32_t spm = 0;
  #pragma unroll
        for (int k = 0; k < F; ++k) {
          float z[3], r;
          if constexpr (kVol) {
            const float tp = xv.mf[0] * wt[k].y + xv.mf[1] * wt[k].z + xv.mf[2] * wt[k].w;
            const float ure = wt[k].x * gre + tp * gv.y;
            const float uim = wt[k].x * gim - tp * gv.x;
            c32 Fv;
            if (pair_adjoint_t<true>(xv, geom[k], ure, uim, z, r, Fv))
              bwd_accumulate<true>(tacc[k], z, gre * Fv.x + gim * Fv.y, xv.mf,
                                   gv.y * Fv.x - gv.x * Fv.y);
            else
              spm |= 1u << k;
          } else {
            if (pair_adjoint(xv, geom[k], gre, gim, z, r))
              bwd_accumulate<false>(tacc[k], z, r, xv.mf, 0.f);
            else
              spm |= 1u << k;
          }
        }
        if (spm) {
  #pragma unroll
          for (int k = 0; k < F; ++k) {
            if ((spm >> k) & 1u) {
              float z[3], r;
              if constexpr (kVol) {
                const float tp = xv.mf[0] * wt[k].y + xv.mf[1] * wt[k].z + xv.mf[2] * wt[k].w;
                const float ure = wt[k].x * gre + tp * gv.y;
                const float uim = wt[k].x * gim - tp * gv.x;
                c32 Fv;
                pair_adjoint_degenerate(xv, geom[k], ure, uim, z, r, Fv);
                bwd_accumulate<true>(tacc[k], z, gre * Fv.x + gim * Fv.y, xv.mf,
                                     gv.y * Fv.x - gv.x * Fv.y);
              } else {
                pair_adjoint_degenerate(xv, geom[k], gre, gim, z, r);
                bwd_accumulate<false>(tacc[k], z, r, xv.mf, 0.f);
              }
            }
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < F; ++k)
#pragma unroll
      for (int i = 0; i < NQ; ++i) acc[k].q[i] += tacc[k].q[i];
    __syncthreads();
    if (threadIdx.x == 0 && t + NS < ntiles) {
      fence_proxy_async();
      const int tn = t + NS;
      stage_tile<kVol>(&sx[s][0], &sg[kVol ? s : 0][0], src0, xg + d.b_off + x0, tn * TX,
                       min(TX, nx - tn * TX), &bar[s]);
    }
  }
  float* out = bpart + d.bpart_off + (int64_t)chunk * NQ * d.nt;
#pragma unroll
  for (int k = 0; k < F; ++k) {
    if (fidx[k] < d.nt) {
#pragma unroll
      for (int i = 0; i < NQ; ++i) out[(int64_t)i * d.nt + fidx[k]] = acc[k].q[i];
    }
  }
}

}  // namespace dm
