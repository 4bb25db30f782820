// Surface + enclosed-volume ("autofluorescence") transform and its adjoint,
// fourier_from_mesh_narrowband_autofluorescence of deltamic/render.py:228-318:
//
//   ft(xi) = sum_k F_k(xi) (a_k + i beta (xi . nor_k) / |xi|^2),
//   a_k = 2 A_k / sum_j A_j          (render.py:202-218, 235-236; no Faces_coeff)
//   nor_k = p0 x p1 + p1 x p2 + p2 x p0        (render.py:217)
//   beta = regint / regvol, regvol = -sum_k p0 . (p1 x p2) / 6   (render.py:221-232)
//
// with F the per-pair term of the surface transform (pair_math.cuh).  The second
// term is, by the divergence theorem, -beta times the transform of the enclosed
// volume with the normals' orientation; its value at xi = 0 (a grid with every
// axis odd) is 0/0 in the reference (NaN) and is taken here as its limit,
// -regint.  Vertex coordinates enter as given (the reference does not shift them
// into the box): the caller passes a box with lower corner 0.
//
// One F evaluation per pair feeds both sums: the main kernels of the surface
// transform run with kVol set (meshft_kernels.cuh).  The forward also returns
// vol(xi) = i sum_k F_k (xi . nor_k) / |xi|^2 (ft = surface + beta vol), which the
// backward needs for the regint and regvol terms.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "dm_common.cuh"
#include "meshft_internal.h"
#include "meshft_kernels.cuh"
#include "pair_math.cuh"

namespace dm {
namespace {

// Tile shapes of the fit step's tuned surface kernels at 200^3 (forward {2, 256},
// adjoint {1, 128}, 16 items per SM).
constexpr int kVolR = 2, kVolFwdNT = 256;  // forward: frequencies per thread, threads
constexpr int kVolF = 1, kVolBwdNT = 128;  // adjoint: faces per thread, threads
constexpr int kVolWaves = 16;
constexpr int kVolQ = 13;                  // adjoint accumulators per face
constexpr double kPi = 3.141592653589793;

Cells single(const CellDesc& d) {
  Cells c;
  c.p = nullptr;
  c.n = 1;
  c.one = d;
  return c;
}

int status() { return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA; }

struct VolScalars {
  double M, regvol, beta;
};

// Sum of face areas, regvol and beta, identical in every block (fixed order).
__device__ VolScalars vol_scalars(const CellDesc& d, const double* area_part,
                                  const double* det_part, const float* regint, double* sh) {
  const int nb = (d.nt + kBlk - 1) / kBlk;
  VolScalars s;
  s.M = block_sum_list(area_part, nb, sh);
  s.regvol = -block_sum_list(det_part, nb, sh) / 6.0;
  s.beta = d.nt > 0 ? (double)*regint / s.regvol : 0.0;  // no faces: ft = 0
  return s;
}

__device__ __forceinline__ void load_face(const CellDesc& d, const float* verts,
                                          const int64_t* faces, int f, double P[3][3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    int64_t v = faces[3 * (int64_t)f + k];
    if (v < 0 || v >= d.nv) v = 0;  // flagged by k_face_prep
#pragma unroll
    for (int j = 0; j < 3; ++j) P[k][j] = (double)verts[3 * v + j];
  }
}

__device__ __forceinline__ void cross3(const double a[3], const double b[3], double c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// |xi|^2 of a grid frequency (integer offsets m) and whether it is xi = 0.
__device__ __forceinline__ double xi_norm2(const CellDesc& d, const int32_t mi[3], bool& zero) {
  zero = mi[0] == 0 && mi[1] == 0 && mi[2] == 0;
  double q = 0.0;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const double x = (double)mi[j] * kPi / d.len[j];
    q += x * x;
  }
  return q;
}

// vrec[f] = nor_f * pi / L (so m . vrec = xi . nor) and per-block sums of
// p0 . (p1 x p2).
__global__ void k_vol_face_prep(CellDesc d, const float* __restrict__ verts,
                                const int64_t* __restrict__ faces, float4* __restrict__ vrec,
                                double* __restrict__ det_part) {
  __shared__ double sh[40];
  const int f = blockIdx.x * kBlk + threadIdx.x;
  double det = 0.0;
  if (f < d.nt) {
    double P[3][3], c01[3], c12[3], c20[3];
    load_face(d, verts, faces, f, P);
    cross3(P[0], P[1], c01);
    cross3(P[1], P[2], c12);
    cross3(P[2], P[0], c20);
    det = P[0][0] * c12[0] + P[0][1] * c12[1] + P[0][2] * c12[2];
    float4 r;
    r.x = (float)((c01[0] + c12[0] + c20[0]) * kPi / d.len[0]);
    r.y = (float)((c01[1] + c12[1] + c20[1]) * kPi / d.len[1]);
    r.z = (float)((c01[2] + c12[2] + c20[2]) * kPi / d.len[2]);
    r.w = 0.f;
    vrec[f] = r;
  }
  const double s = block_sum_d(det, sh);
  if (threadIdx.x == 0) det_part[blockIdx.x] = s;
}

// ft = (2/M) surface sum + beta vol, vol = i (volume sum) / |xi|^2 (-regvol at
// xi = 0); mirror entries conj; optional scatter of ft * OTF into the grid.
__global__ void k_vol_fwd_epi(CellDesc d, const int32_t* __restrict__ band_index,
                              const float2* __restrict__ fpart,
                              const double* __restrict__ area_part,
                              const double* __restrict__ det_part, const float* regint,
                              const float* __restrict__ otf, float2* __restrict__ ft_list,
                              float2* __restrict__ vol_list, float2* __restrict__ grid,
                              int* err) {
  __shared__ double sh[40];
  const VolScalars sc = vol_scalars(d, area_part, det_part, regint, sh);
  const int m = blockIdx.x * kBlk + threadIdx.x;
  if (m >= d.ne) return;
  double sx = 0.0, sy = 0.0, vx = 0.0, vy = 0.0;
  const float2* pa = fpart + m;
  const float2* pb = fpart + (int64_t)d.fsplit * d.ne + m;
  int s = 0;
  for (; s + 4 <= d.fsplit; s += 4) {  // eight loads in flight, summed in split order
    float2 a[4], b[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a[u] = pa[(int64_t)(s + u) * d.ne];
      b[u] = pb[(int64_t)(s + u) * d.ne];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      sx += a[u].x;
      sy += a[u].y;
      vx += b[u].x;
      vy += b[u].y;
    }
  }
  for (; s < d.fsplit; ++s) {
    const float2 a = pa[(int64_t)s * d.ne], b = pb[(int64_t)s * d.ne];
    sx += a.x;
    sy += a.y;
    vx += b.x;
    vy += b.y;
  }
  const int64_t nvox = (int64_t)d.n[0] * d.n[1] * d.n[2];
  const int mr = d.nband - 1 - m;
  const bool mirror = d.herm && mr != m;
  const int32_t idx = band_index[m];
  const int32_t idr = mirror ? band_index[mr] : idx;
  const bool ok = idx >= 0 && (int64_t)idx < nvox &&
                  (!mirror || (int64_t)idr == nvox - 1 - (int64_t)idx);
  if (!ok) {
    set_error(err, DM_ERR_BAD_INDEX);
    return;
  }
  int32_t mi[3];
  band_to_m(idx, d, mi);
  bool zero;
  const double q = xi_norm2(d, mi, zero);
  double wx = zero ? -sc.regvol : -vy / q, wy = zero ? 0.0 : vx / q;
  double fx = 2.0 * sx / sc.M + sc.beta * wx, fy = 2.0 * sy / sc.M + sc.beta * wy;
  if (d.nt == 0) fx = fy = wx = wy = 0.0;  // no faces: ft = 0
  const float2 ft = make_float2((float)fx, (float)fy);
  const float2 vol = make_float2((float)wx, (float)wy);
  ft_list[m] = ft;
  vol_list[m] = vol;
  if (mirror) {
    ft_list[mr] = make_float2(ft.x, -ft.y);
    vol_list[mr] = make_float2(vol.x, -vol.y);
  }
  if (grid) {
    const float o = otf ? otf[idx] : 1.0f;
    grid[idx] = make_float2(ft.x * o, ft.y * o);
    if (mirror) {
      const float orr = otf ? otf[idr] : 1.0f;
      grid[idr] = make_float2(ft.x * orr, -ft.y * orr);
    }
  }
}

// Band records for the adjoint: XiRec with the (mirror-folded) cotangent g,
// xg = g / |xi|^2 (0 at xi = 0), and per-block sums over the whole band of
//   s_part[0][b] = Re(conj(g) (ft - beta vol))   (surface part)
//   s_part[1][b] = Re(conj(g) vol), xi != 0      (d loss / d beta)
//   s_part[2][b] = Re(g) at xi = 0               (ft(0) = surface - regint)
__global__ void k_vol_band_prep(CellDesc d, const int32_t* __restrict__ band_index,
                                const float2* __restrict__ grad_list,
                                const float2* __restrict__ grad_grid,
                                const float* __restrict__ otf, float grad_scale,
                                const float2* __restrict__ ft_list,
                                const float2* __restrict__ vol_list,
                                const double* __restrict__ area_part,
                                const double* __restrict__ det_part, const float* regint,
                                XiRec* __restrict__ xrec, float4* __restrict__ xg,
                                double* __restrict__ s_part, int band_blks, int* err) {
  __shared__ double sh[40];
  const VolScalars sc = vol_scalars(d, area_part, det_part, regint, sh);
  const int m = blockIdx.x * kBlk + threadIdx.x;
  const int64_t nvox = (int64_t)d.n[0] * d.n[1] * d.n[2];
  double sa = 0.0, gb = 0.0, g0 = 0.0;
  if (m < d.nband) {
    int32_t idx = band_index[m];
    const bool ok = idx >= 0 && (int64_t)idx < nvox;
    if (!ok) {
      set_error(err, DM_ERR_BAD_INDEX);
      idx = 0;
    }
    float2 G;
    float2 g = band_cotangent(d, m, idx, ok, grad_list, grad_grid, otf, grad_scale, G);
    const float2 ft = ft_list[m], vol = vol_list[m];
    int32_t mi[3];
    band_to_m(idx, d, mi);
    bool zero;
    const double q = xi_norm2(d, mi, zero);
    sa = (double)g.x * ((double)ft.x - sc.beta * vol.x) +
         (double)g.y * ((double)ft.y - sc.beta * vol.y);
    if (zero)
      g0 = g.x;
    else
      gb = (double)g.x * vol.x + (double)g.y * vol.y;
    if (m < d.ne) {
      const int mr = d.nband - 1 - m;
      if (d.herm && mr != m) {
        int32_t idr = band_index[mr];
        const bool okr = ok && (int64_t)idr == nvox - 1 - (int64_t)idx;
        if (!okr) {
          set_error(err, DM_ERR_BAD_INDEX);
          idr = 0;
        }
        float2 Gr;
        const float2 gr = band_cotangent(d, mr, idr, okr, grad_list, grad_grid, otf,
                                         grad_scale, Gr);
        g.x += gr.x;
        g.y -= gr.y;
      }
      XiRec r;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        r.mi[k] = mi[k];
        r.mf[k] = (float)mi[k];
      }
      r.g_re = g.x;
      r.g_im = g.y;
      xrec[m] = r;
      const double iq = zero ? 0.0 : 1.0 / q;
      xg[m] = make_float4((float)(g.x * iq), (float)(g.y * iq), 0.f, 0.f);
    }
  }
  const double t0 = block_sum_d(sa, sh);
  const double t1 = block_sum_d(gb, sh);
  const double t2 = block_sum_d(g0, sh);
  if (threadIdx.x == 0) {
    s_part[blockIdx.x] = t0;
    s_part[band_blks + blockIdx.x] = t1;
    s_part[2 * band_blks + blockIdx.x] = t2;
  }
}

// Per-face weights of the adjoint: fw[f] = {2 A_f / M, beta nor'_f}.
__global__ void k_vol_face_weights(CellDesc d, const FaceRec* __restrict__ recs,
                                   const float4* __restrict__ vrec,
                                   const double* __restrict__ area_part,
                                   const double* __restrict__ det_part, const float* regint,
                                   float4* __restrict__ fw) {
  __shared__ double sh[40];
  const VolScalars sc = vol_scalars(d, area_part, det_part, regint, sh);
  const int f = blockIdx.x * kBlk + threadIdx.x;
  if (f >= d.nt) return;
  const float4 v = vrec[f];
  fw[f] = make_float4((float)(2.0 * recs[f].area_coeff / sc.M), (float)(sc.beta * v.x),
                      (float)(sc.beta * v.y), (float)(sc.beta * v.z));
}

// Per-face epilogue: reduce the chunks' 13 sums, then per corner v of face f
//   contrib = (pi/L) Q_v + dL/dA dA/dp_v + beta (p_next - p_prev) x N'
//             + dL/dregvol (-(p_next x p_prev) / 6)
// with dL/dA = (2 r - S_A)/M, N' = (pi/L) * the normal sums, dL/dregvol =
// -G_beta beta / regvol; block 0 writes dL/dregint = G_beta / regvol - Re(g(0)).
__global__ void k_vol_face_epi(CellDesc d, const float* __restrict__ verts,
                               const int64_t* __restrict__ faces,
                               const double* __restrict__ area_part,
                               const double* __restrict__ det_part,
                               const double* __restrict__ s_part, int band_blks,
                               const float* regint, const float* __restrict__ bpart,
                               float* __restrict__ contrib, float* __restrict__ grad_regint) {
  __shared__ double sh[40];
  const VolScalars sc = vol_scalars(d, area_part, det_part, regint, sh);
  const double SA = block_sum_list(s_part, band_blks, sh);
  const double GB = block_sum_list(s_part + band_blks, band_blks, sh);
  const double G0 = block_sum_list(s_part + 2 * band_blks, band_blks, sh);
  if (blockIdx.x == 0 && threadIdx.x == 0 && grad_regint)
    *grad_regint = d.nt > 0 ? (float)(GB / sc.regvol - G0) : 0.f;
  const int f = blockIdx.x * kBlk + threadIdx.x;
  if (f >= d.nt) return;
  double q[kVolQ];
#pragma unroll
  for (int i = 0; i < kVolQ; ++i) q[i] = 0.0;
  int c = 0;
  for (; c + 2 <= d.bchunks; c += 2) {  // 26 loads in flight, summed in chunk order
    float v[2][kVolQ];
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int i = 0; i < kVolQ; ++i) v[u][i] = bpart[((int64_t)(c + u) * kVolQ + i) * d.nt + f];
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int i = 0; i < kVolQ; ++i) q[i] += v[u][i];
  }
  for (; c < d.bchunks; ++c) {
#pragma unroll
    for (int i = 0; i < kVolQ; ++i) q[i] += bpart[((int64_t)c * kVolQ + i) * d.nt + f];
  }
  double P[3][3];
  load_face(d, verts, faces, f, P);
  const double e1[3] = {P[1][0] - P[0][0], P[1][1] - P[0][1], P[1][2] - P[0][2]};
  const double e2[3] = {P[2][0] - P[0][0], P[2][1] - P[0][1], P[2][2] - P[0][2]};
  double n[3];
  cross3(e1, e2, n);
  const double nn = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  n[0] /= nn;
  n[1] /= nn;
  n[2] /= nn;
  const double dlda = (2.0 * q[9] - SA) / sc.M;
  const double dlrv = -GB * sc.beta / sc.regvol;
  double xs[3], Nn[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    xs[j] = kPi / d.len[j];
    Nn[j] = q[10 + j] * xs[j];
  }
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    const double* pn = P[v == 2 ? 0 : v + 1];
    const double* pp = P[v == 0 ? 2 : v - 1];
    const double e[3] = {pp[0] - pn[0], pp[1] - pn[1], pp[2] - pn[2]};
    const double dv[3] = {-e[0], -e[1], -e[2]};  // p_next - p_prev
    double dA[3], dn[3], pc[3];
    cross3(n, e, dA);
    cross3(dv, Nn, dn);
    cross3(pn, pp, pc);
#pragma unroll
    for (int j = 0; j < 3; ++j)
      contrib[9 * (int64_t)f + 3 * v + j] =
          (float)(xs[j] * q[3 * v + j] + dlda * 0.5 * dA[j] + sc.beta * dn[j] -
                  dlrv * pc[j] / 6.0);
  }
}

int64_t cdiv64(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace

void plan_volume(CellDesc& d, PlanTotals& t) {
  plan_cell_tiles_for(d, FwdVariant{kVolR, kVolFwdNT, kVolWaves},
                      BwdVariant{kVolF, kVolBwdNT, kVolWaves});
  t.fpart = 2 * (int64_t)d.fsplit * d.ne;
  t.bpart = (int64_t)kVolQ * d.bchunks * d.nt;
  t.fwd_items = (int64_t)d.xtiles * d.fsplit;
  t.bwd_items = (int64_t)d.fblocks * d.bchunks;
}

int launch_volume_forward(const CellDesc& d, const PlanTotals& t, const float* verts,
                          const int64_t* faces, const float* regint, const int32_t* band_index,
                          const float* otf, double* area_part, double* det_part, FaceRec* recs,
                          float4* vrec, float2* fpart, float2* ft_list, float2* vol_list,
                          float2* grid, int* err, cudaStream_t st) {
  const Cells c = single(d);
  int s = launch_face_prep(c, t, verts, faces, nullptr, recs, area_part, err, st);
  if (s) return s;
  k_vol_face_prep<<<(unsigned)t.face_blks, kBlk, 0, st>>>(d, verts, faces, vrec, det_part);
  count_launches(1);
  if (status()) return DM_ERR_CUDA;
  if (t.nband <= 0) return DM_OK;
  if (t.fwd_items > 0) {
    profile_begin(0, st);
    k_meshft_fwd<kVolR, kVolFwdNT, kFwdTF, kStages, true>
        <<<(unsigned)t.fwd_items, kVolFwdNT, 0, st>>>(c, recs, vrec, band_index, nullptr, fpart, err);
    profile_end(0, st);
    count_launches(1);
    if (status()) return DM_ERR_CUDA;
  }
  k_vol_fwd_epi<<<(unsigned)std::max<int64_t>(1, cdiv64(d.ne, kBlk)), kBlk, 0, st>>>(
      d, band_index, fpart, area_part, det_part, regint, otf, ft_list, vol_list, grid, err);
  count_launches(1);
  return status();
}

int launch_volume_backward(const CellDesc& d, const PlanTotals& t, const float* verts,
                           const int64_t* faces, const float* regint, const int32_t* band_index,
                           const float2* grad_list, const float2* grad_grid, const float* otf,
                           float grad_scale, const float2* ft_list, const float2* vol_list,
                           double* area_part, double* det_part, double* s_part, FaceRec* recs,
                           float4* vrec, float4* fw, XiRec* xrec, float4* xg, float* bpart,
                           float* contrib, const int32_t* csr_off, const int32_t* csr_ent,
                           float* grad_verts, float* grad_regint, int* err, cudaStream_t st) {
  const Cells c = single(d);
  int s = launch_face_prep(c, t, verts, faces, nullptr, recs, area_part, err, st);
  if (s) return s;
  const unsigned fb = (unsigned)t.face_blks, bb = (unsigned)t.band_blks;
  k_vol_face_prep<<<fb, kBlk, 0, st>>>(d, verts, faces, vrec, det_part);
  k_vol_face_weights<<<fb, kBlk, 0, st>>>(d, recs, vrec, area_part, det_part, regint, fw);
  k_vol_band_prep<<<bb, kBlk, 0, st>>>(d, band_index, grad_list, grad_grid, otf, grad_scale,
                                       ft_list, vol_list, area_part, det_part, regint, xrec, xg,
                                       s_part, (int)t.band_blks, err);
  count_launches(3);
  if (status()) return DM_ERR_CUDA;
  cudaMemsetAsync(bpart, 0, sizeof(float) * (size_t)std::max<int64_t>(t.bpart, 1), st);
  if (t.bwd_items > 0 && t.nband > 0 && t.nt > 0) {
    profile_begin(1, st);
    k_meshft_bwd<kVolF, kVolBwdNT, kBwdTX, kStages, true>
        <<<(unsigned)t.bwd_items, kVolBwdNT, 0, st>>>(c, recs, fw, xrec, xg, nullptr, bpart, err);
    profile_end(1, st);
    count_launches(1);
    if (status()) return DM_ERR_CUDA;
  }
  k_vol_face_epi<<<fb, kBlk, 0, st>>>(d, verts, faces, area_part, det_part, s_part,
                                      (int)t.band_blks, regint, bpart, contrib, grad_regint);
  count_launches(1);
  if (status()) return DM_ERR_CUDA;
  return launch_vertex_gather(t.nv, csr_off, csr_ent, contrib, grad_verts, st);
}

}  // namespace dm
