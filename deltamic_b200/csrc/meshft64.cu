// Float64 meshFT: forward and adjoint in double precision with the reference's
// float64 CPU arithmetic (MeshFTPy, deltamic/render.py:36-109, whose Seps is
// sqrt(1.19209e-07) for both dtypes, render.py:64-65, with a strict comparison in
// R1 and <= in R2-R4, :77-82), and the partials of the CUDA path
// (deltamic/cpp/fourier3d_cuda_kernel.cu:73-233, adjoint :314-416).
//
// Per (face, frequency) pair with vertex phases x_v = xi . v (double):
//   F = e_a w_a + e_b w_b + e_c w_c,  e_v = exp(-i x_v),
//   w_a = 1/(ab ca), w_b = 1/(bc ab), w_c = 1/(ca bc)  (ab = x_b - x_a, ...),
// the minus second divided difference of exp(-i x), with the reference's
// branches when a difference is within Seps: R1 (two of them) the centroid value
// e^{-i mean}/2, R2/R3/R4 the close pair merged at its midpoint d:
// F = (i e_d + (e_d - e_o)/D)/D, D = d - x_o.  The partials are the derivatives of
// those same expressions (merged vertices share dF/dd / 2; R1 gives -iF/3 each).
//
// Why the CPU path's Seps and not the CUDA double dispatch's sqrt(DBL_EPSILON)
// (.cu:454, :522): the general formula cancels ~1/D^2 (F) and ~1/D^3 (partials)
// terms, so with differences D between 1.5e-8 and ~1e-5 it loses the partials to
// rounding (measured here: 2e-4 rel-L2 on a level-4 vertex gradient against the
// CPU float64 reference, and 3e-4 on the spectrum at |xi| ~ 1e-5).  Above
// 3.45e-4 the rounding error of the partials stays below ~3e-6 of their size.
//
// Layout and work split follow the float32 kernels: face records (80 B) and
// frequency records (48 B) staged in shared memory by bulk copies into a ring of
// mbarrier-completed tiles; forward item = (frequency tile, face split) with the
// split partials summed in a fixed order; adjoint item = (face block, frequency
// chunk) with per-face partials summed in a fixed order, then the vertex <- face
// CSR gather.  Deterministic, no atomics.  Two frequency sources: the centred
// grid of a box (band voxel indices; vertices shifted by box.lo as
// Fourier3dMesh.forward does) or an explicit xi list (vertices as given, the
// forward_fourier3d_cpp convention).  Every frequency is evaluated (no mirror).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>

#include "dm_common.cuh"
#include "meshft_internal.h"
#include "meshft_kernels.cuh"

namespace dm {

namespace {

constexpr double kSeps64 = 3.4526656368666803e-04;  // sqrt(1.19209e-07), render.py:64-65
constexpr int kBlk64 = 256;  // element-wise kernels
constexpr int kNT64 = 128;   // threads of the main kernels
constexpr int kTF64 = 64;    // faces per staged tile (forward), = kFwdTF
constexpr int kTX64 = 128;   // frequencies per staged tile (adjoint), = kBwdTX
constexpr int kNS64 = 3;     // stages of the ring

struct alignas(16) Face64 {
  double v[9];  // a, b, c (shifted by the box's lower corner in grid mode)
  double ac;    // |(b-a)x(c-a)|/2 * Faces_coeff
};
static_assert(sizeof(Face64) == 80, "Face64 layout");

struct alignas(16) Xi64 {
  double xi[3];
  double g_re, g_im;  // adjoint cotangent (0 in the forward)
  double pad;
};
static_assert(sizeof(Xi64) == 48, "Xi64 layout");

struct cd {
  double x, y;
};

__device__ __forceinline__ cd emi(double x) {
  double s, c;
  sincos(x, &s, &c);
  return cd{c, -s};
}
__device__ __forceinline__ cd cadd(cd a, cd b) { return cd{a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cd csc(double s, cd a) { return cd{s * a.x, s * a.y}; }
__device__ __forceinline__ cd cmulx(cd a, cd b) {
  return cd{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
__device__ __forceinline__ cd cdivr(cd a, double r) { return cd{a.x / r, a.y / r}; }
__device__ __forceinline__ cd mul_i(cd a) { return cd{-a.y, a.x}; }      // i a
__device__ __forceinline__ cd mul_mi(cd a) { return cd{a.y, -a.x}; }     // -i a

// Branch of a pair: 0 = R5 (general), 1 = R1, 2/3/4 = R2/R3/R4.
__device__ __forceinline__ int branch64(double ab, double bc, double ca) {
  const bool tab = fabs(ab) < kSeps64, tbc = fabs(bc) < kSeps64, tca = fabs(ca) < kSeps64;
  if ((tab && tbc) || (tbc && tca) || (tca && tab)) return 1;
  const bool sab = fabs(ab) <= kSeps64, sbc = fabs(bc) <= kSeps64, sca = fabs(ca) <= kSeps64;
  if (sab) return 2;
  if (sbc) return 3;
  if (sca) return 4;
  return 0;
}

// F and, with kGrad, dF/dx_{a,b,c} at phases xa, xb, xc.
template <bool kGrad>
__device__ __forceinline__ cd pair64(double xa, double xb, double xc, cd* dF) {
  const double ab = xb - xa, bc = xc - xb, ca = xa - xc;
  const int br = branch64(ab, bc, ca);
  if (br == 0) {
    const cd ea = emi(xa), eb = emi(xb), ec = emi(xc);
    const double iab = 1.0 / ab, ibc = 1.0 / bc, ica = 1.0 / ca;
    const double wa = iab * ica, wb = ibc * iab, wc = ica * ibc;
    const cd F = cadd(cadd(csc(wa, ea), csc(wb, eb)), csc(wc, ec));
    if (kGrad) {
      // d/dx_a [e_a w_a] = e_a w_a (iab - ica - i); d/dx_a [e_b w_b] = e_b w_b iab;
      // d/dx_a [e_c w_c] = -e_c w_c ica; and cyclically for b and c.
      const cd ta = csc(wa, ea), tb = csc(wb, eb), tc = csc(wc, ec);
      dF[0] = cadd(cadd(cadd(csc(iab - ica, ta), mul_mi(ta)), csc(iab, tb)), csc(-ica, tc));
      dF[1] = cadd(cadd(cadd(csc(ibc - iab, tb), mul_mi(tb)), csc(ibc, tc)), csc(-iab, ta));
      dF[2] = cadd(cadd(cadd(csc(ica - ibc, tc), mul_mi(tc)), csc(ica, ta)), csc(-ibc, tb));
    }
    return F;
  }
  if (br == 1) {
    const cd F = csc(0.5, emi((xa + xb + xc) / 3.0));
    if (kGrad) {
      const cd g = csc(1.0 / 3.0, mul_mi(F));
      dF[0] = dF[1] = dF[2] = g;
    }
    return F;
  }
  // merged pair (p, q) at d, lone vertex o
  double d, xo;
  int o;
  if (br == 2) {
    d = (xa + xb) / 2.0;
    xo = xc;
    o = 2;
  } else if (br == 3) {
    d = (xb + xc) / 2.0;
    xo = xa;
    o = 0;
  } else {
    d = (xc + xa) / 2.0;
    xo = xb;
    o = 1;
  }
  const cd ed = emi(d), eo = emi(xo);
  const double D = d - xo;
  const cd F = cdivr(cadd(mul_i(ed), cdivr(cd{ed.x - eo.x, ed.y - eo.y}, D)), D);
  if (kGrad) {
    // dF/dx of each merged vertex: (dF/dd)/2 = (e_d/2 - F)/D; the lone vertex
    // gets -iF - 2 of that (the three partials sum to -iF, translation)
    const cd gm = cdivr(cd{0.5 * ed.x - F.x, 0.5 * ed.y - F.y}, D);
    const cd go = cadd(mul_mi(F), csc(-2.0, gm));
    dF[0] = dF[1] = dF[2] = gm;
    dF[o] = go;
  }
  return F;
}

__device__ __forceinline__ double dot3(const double* v, const double* x) {
  return v[0] * x[0] + v[1] * x[1] + v[2] * x[2];
}

__device__ __forceinline__ double block_sum64(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)((blockDim.x + 31) >> 5); ++i) r += sh[i];
  __syncthreads();
  return r;
}

__device__ __forceinline__ double sum_list64(const double* p, int n, double* sh) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += p[i];
  double r = block_sum64(v, sh);
  if (threadIdx.x == 0) sh[32] = r;
  __syncthreads();
  r = sh[32];
  __syncthreads();
  return r;
}

// ---------------------------------------------------------------------------

__global__ void k64_face_prep(CellDesc d, const double* __restrict__ verts,
                              const int64_t* __restrict__ faces,
                              const double* __restrict__ coeff, Face64* __restrict__ recs,
                              double* __restrict__ area_part, int* err) {
  __shared__ double sh[40];
  const int f = blockIdx.x * kBlk64 + threadIdx.x;
  double ac = 0.0;
  if (f < d.nt) {
    int64_t iv[3];
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      iv[k] = faces[3 * (int64_t)f + k];
      if (iv[k] < 0 || iv[k] >= d.nv) {
        ok = false;
        iv[k] = 0;
      }
    }
    if (!ok) set_error(err, DM_ERR_BAD_INDEX);
    Face64 r;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int j = 0; j < 3; ++j) r.v[3 * k + j] = verts[3 * iv[k] + j] - d.lo[j];
    const double e1[3] = {r.v[3] - r.v[0], r.v[4] - r.v[1], r.v[5] - r.v[2]};
    const double e2[3] = {r.v[6] - r.v[0], r.v[7] - r.v[1], r.v[8] - r.v[2]};
    const double cx = e1[1] * e2[2] - e1[2] * e2[1];
    const double cy = e1[2] * e2[0] - e1[0] * e2[2];
    const double cz = e1[0] * e2[1] - e1[1] * e2[0];
    ac = 0.5 * sqrt(cx * cx + cy * cy + cz * cz) * coeff[f];
    r.ac = ac;
    recs[f] = r;
  }
  const double s = block_sum64(ac, sh);
  if (threadIdx.x == 0) area_part[blockIdx.x] = s;
}

// Frequency records: xi from the grid (band voxel index -> m pi / L) or the list;
// with a cotangent (adjoint), g = grad_scale G (otf), and per-block sums of
// s = Re(conj(g) ft) over the list.
__global__ void k64_xi_prep(CellDesc d, const int32_t* __restrict__ band_index,
                            const double* __restrict__ xi_list,
                            const double2* __restrict__ grad_list,
                            const double2* __restrict__ grad_grid,
                            const double* __restrict__ otf, double grad_scale,
                            const double2* __restrict__ ft_list, Xi64* __restrict__ xr,
                            double* __restrict__ s_part, int* err) {
  __shared__ double sh[40];
  const int m = blockIdx.x * kBlk64 + threadIdx.x;
  double s = 0.0;
  if (m < d.nband) {
    Xi64 r;
    int32_t idx = 0;
    bool ok = true;
    if (band_index) {
      const int64_t nvox = (int64_t)d.n[0] * d.n[1] * d.n[2];
      idx = band_index[m];
      if (idx < 0 || (int64_t)idx >= nvox) {
        set_error(err, DM_ERR_BAD_INDEX);
        ok = false;
        idx = 0;
      }
      const int32_t n12 = d.n[1] * d.n[2];
      const int32_t k[3] = {idx / n12, (idx % n12) / d.n[2], idx % d.n[2]};
#pragma unroll
      for (int j = 0; j < 3; ++j)
        r.xi[j] = (double)(2 * k[j] - (d.n[j] - 1)) * (3.141592653589793 / d.len[j]);
    } else {
#pragma unroll
      for (int j = 0; j < 3; ++j) r.xi[j] = xi_list[3 * (int64_t)m + j];
    }
    r.g_re = r.g_im = r.pad = 0.0;
    if (ok && (grad_list || grad_grid)) {
      const double2 G = grad_list ? grad_list[m] : grad_grid[idx];
      const double sc = grad_scale * (otf ? otf[idx] : 1.0);
      r.g_re = sc * G.x;
      r.g_im = sc * G.y;
      const double2 ft = ft_list[m];
      s = r.g_re * ft.x + r.g_im * ft.y;
    }
    xr[m] = r;
  }
  if (s_part) {
    const double t = block_sum64(s, sh);
    if (threadIdx.x == 0) s_part[blockIdx.x] = t;
  }
}

// fpart[split][m] = sum over the split's faces of ac F(xi_m).
template <int R>
__global__ void __launch_bounds__(kNT64) k64_fwd(CellDesc d, const Face64* __restrict__ recs,
                                                const Xi64* __restrict__ xr,
                                                double2* __restrict__ fpart, int* err) {
  __shared__ __align__(128) Face64 sf[kNS64][kTF64];
  __shared__ __align__(8) uint64_t bar[kNS64];
  const int xt = blockIdx.x % d.xtiles;
  const int split = blockIdx.x / d.xtiles;
  const int f0 = split * d.fchunk;
  const int nf = min(d.nt, f0 + d.fchunk) - f0;
  if (d.nband <= 0) return;
  double xi[R][3];
  int mloc[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int m = xt * kNT64 * R + r * kNT64 + threadIdx.x;
    mloc[r] = m;
    const Xi64 x = xr[min(m, d.nband - 1)];
    xi[r][0] = x.xi[0];
    xi[r][1] = x.xi[1];
    xi[r][2] = x.xi[2];
  }
  cd acc[R];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r] = cd{0.0, 0.0};
  if (nf > 0) {
    const int ntiles = (nf + kTF64 - 1) / kTF64;
    const Face64* src = recs + f0;
    if (threadIdx.x == 0) {
      for (int s = 0; s < kNS64; ++s) mbar_init(&bar[s], 1);
      fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int s = 0; s < kNS64 && s < ntiles; ++s)
        stage_tile<false>(&sf[s][0], (float4*)nullptr, src, (const float4*)nullptr, s * kTF64,
                          min(kTF64, nf - s * kTF64), &bar[s]);
    for (int t = 0; t < ntiles; ++t) {
      const int s = t % kNS64;
      if (!mbar_wait_bounded(&bar[s], (uint32_t)((t / kNS64) & 1), err)) return;
      const int nft = min(kTF64, nf - t * kTF64);
      for (int j = 0; j < nft; ++j) {
        const Face64& fr = sf[s][j];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const cd F = pair64<false>(dot3(&fr.v[0], xi[r]), dot3(&fr.v[3], xi[r]),
                                     dot3(&fr.v[6], xi[r]), nullptr);
          acc[r].x += fr.ac * F.x;
          acc[r].y += fr.ac * F.y;
        }
      }
      __syncthreads();
      if (threadIdx.x == 0 && t + kNS64 < ntiles) {
        fence_proxy_async();
        const int tn = t + kNS64;
        stage_tile<false>(&sf[s][0], (float4*)nullptr, src, (const float4*)nullptr, tn * kTF64,
                          min(kTF64, nf - tn * kTF64), &bar[s]);
      }
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r)
    if (mloc[r] < d.nband)
      fpart[(int64_t)split * d.nband + mloc[r]] = make_double2(acc[r].x, acc[r].y);
}

// ft_list = (2/M) sum over splits (fixed order); optional grid scatter of ft * otf.
__global__ void k64_fwd_epi(CellDesc d, const int32_t* __restrict__ band_index,
                            const double2* __restrict__ fpart,
                            const double* __restrict__ area_part, int n_area,
                            const double* __restrict__ otf, double2* __restrict__ ft_list,
                            double2* __restrict__ grid) {
  __shared__ double sh[40];
  const double M = sum_list64(area_part, n_area, sh);
  const int m = blockIdx.x * kBlk64 + threadIdx.x;
  if (m >= d.nband) return;
  double sx = 0.0, sy = 0.0;
  for (int s = 0; s < d.fsplit; ++s) {
    const double2 v = fpart[(int64_t)s * d.nband + m];
    sx += v.x;
    sy += v.y;
  }
  const double sc = d.nt > 0 ? 2.0 / M : 0.0;
  const double2 ft = make_double2(sx * sc, sy * sc);
  ft_list[m] = ft;
  if (grid && band_index) {
    const int64_t nvox = (int64_t)d.n[0] * d.n[1] * d.n[2];
    const int32_t idx = band_index[m];
    if (idx < 0 || (int64_t)idx >= nvox) return;  // reported by k64_xi_prep
    const double o = otf ? otf[idx] : 1.0;
    grid[idx] = make_double2(ft.x * o, ft.y * o);
  }
}

// bpart[chunk][i][f]: q[3v+j] = sum z_v xi_j, q[9] = sum r over the chunk, with
// z_v = Re(conj(g) dF/dx_v) and r = Re(conj(g) F).
template <int F>
__global__ void __launch_bounds__(kNT64) k64_bwd(CellDesc d, const Face64* __restrict__ recs,
                                                const Xi64* __restrict__ xr,
                                                double* __restrict__ bpart, int* err) {
  __shared__ __align__(128) Xi64 sx[kNS64][kTX64];
  __shared__ __align__(8) uint64_t bar[kNS64];
  const int fb = blockIdx.x % d.fblocks;
  const int chunk = blockIdx.x / d.fblocks;
  const int x0 = chunk * d.bxchunk;
  const int nx = min(d.nband, x0 + d.bxchunk) - x0;
  if (nx <= 0 || d.nt <= 0) return;
  Face64 fr[F];
  int fidx[F];
#pragma unroll
  for (int k = 0; k < F; ++k) {
    const int f = fb * kNT64 * F + k * kNT64 + threadIdx.x;
    fidx[k] = f;
    fr[k] = recs[min(f, d.nt - 1)];
  }
  double q[F][10];
#pragma unroll
  for (int k = 0; k < F; ++k)
#pragma unroll
    for (int i = 0; i < 10; ++i) q[k][i] = 0.0;
  const int ntiles = (nx + kTX64 - 1) / kTX64;
  const Xi64* src = xr + x0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kNS64; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int s = 0; s < kNS64 && s < ntiles; ++s)
      stage_tile<false>(&sx[s][0], (float4*)nullptr, src, (const float4*)nullptr, s * kTX64,
                        min(kTX64, nx - s * kTX64), &bar[s]);
  for (int t = 0; t < ntiles; ++t) {
    const int s = t % kNS64;
    if (!mbar_wait_bounded(&bar[s], (uint32_t)((t / kNS64) & 1), err)) return;
    const int nxt = min(kTX64, nx - t * kTX64);
    for (int j = 0; j < nxt; ++j) {
      const Xi64& x = sx[s][j];
#pragma unroll
      for (int k = 0; k < F; ++k) {
        cd dF[3];
        const cd Fv = pair64<true>(dot3(&fr[k].v[0], x.xi), dot3(&fr[k].v[3], x.xi),
                                   dot3(&fr[k].v[6], x.xi), dF);
#pragma unroll
        for (int v = 0; v < 3; ++v) {
          const double z = x.g_re * dF[v].x + x.g_im * dF[v].y;
          q[k][3 * v + 0] += z * x.xi[0];
          q[k][3 * v + 1] += z * x.xi[1];
          q[k][3 * v + 2] += z * x.xi[2];
        }
        q[k][9] += x.g_re * Fv.x + x.g_im * Fv.y;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && t + kNS64 < ntiles) {
      fence_proxy_async();
      const int tn = t + kNS64;
      stage_tile<false>(&sx[s][0], (float4*)nullptr, src, (const float4*)nullptr, tn * kTX64,
                        min(kTX64, nx - tn * kTX64), &bar[s]);
    }
  }
  double* out = bpart + (int64_t)chunk * 10 * d.nt;
#pragma unroll
  for (int k = 0; k < F; ++k)
    if (fidx[k] < d.nt)
#pragma unroll
      for (int i = 0; i < 10; ++i) out[(int64_t)i * d.nt + fidx[k]] = q[k][i];
}

// Per face: contrib[f][v][j] = trisar Q[v][j] + (c/M)(2r - S) dA/dv_j and
// grad_coeff[f] = (A/M)(2r - S), trisar = 2Ac/M (the reference's adjoint,
// .cu:365-394, with the edge normals and mesh-area gradient folded per face).
__global__ void k64_face_epi(CellDesc d, const Face64* __restrict__ recs,
                             const double* __restrict__ coeff,
                             const double* __restrict__ area_part, int n_area,
                             const double* __restrict__ s_part, int n_s,
                             const double* __restrict__ bpart, double* __restrict__ contrib,
                             double* __restrict__ grad_coeff) {
  __shared__ double sh[40];
  const double M = sum_list64(area_part, n_area, sh);
  const double S = sum_list64(s_part, n_s, sh);
  const int f = blockIdx.x * kBlk64 + threadIdx.x;
  if (f >= d.nt) return;
  double q[10];
#pragma unroll
  for (int i = 0; i < 10; ++i) q[i] = 0.0;
  for (int c = 0; c < d.bchunks; ++c)
#pragma unroll
    for (int i = 0; i < 10; ++i) q[i] += bpart[((int64_t)c * 10 + i) * d.nt + f];
  const Face64 r = recs[f];
  const double* P = r.v;
  const double e1[3] = {P[3] - P[0], P[4] - P[1], P[5] - P[2]};
  const double e2[3] = {P[6] - P[0], P[7] - P[1], P[8] - P[2]};
  double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                 e1[0] * e2[1] - e1[1] * e2[0]};
  const double nn = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  const double A = 0.5 * nn;
  if (nn > 0.0) {
    n[0] /= nn;
    n[1] /= nn;
    n[2] /= nn;
  }
  const double c = coeff[f];
  const double trisar = 2.0 * A * c / M;
  const double k2 = 2.0 * q[9] - S;
  const double kk = (c / M) * k2;
  if (grad_coeff) grad_coeff[f] = (A / M) * k2;
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    const double* pn = &P[3 * ((v + 1) % 3)];
    const double* pp = &P[3 * ((v + 2) % 3)];
    const double e[3] = {pp[0] - pn[0], pp[1] - pn[1], pp[2] - pn[2]};
    const double dA[3] = {0.5 * (n[1] * e[2] - n[2] * e[1]), 0.5 * (n[2] * e[0] - n[0] * e[2]),
                          0.5 * (n[0] * e[1] - n[1] * e[0])};
#pragma unroll
    for (int j = 0; j < 3; ++j)
      contrib[9 * (int64_t)f + 3 * v + j] = trisar * q[3 * v + j] + kk * dA[j];
  }
}

__global__ void k64_vertex_gather(int64_t nv, const int32_t* __restrict__ off,
                                  const int32_t* __restrict__ ent,
                                  const double* __restrict__ contrib, double* __restrict__ gv) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  double g0 = 0.0, g1 = 0.0, g2 = 0.0;
  for (int32_t i = off[v]; i < off[v + 1]; ++i) {
    const int32_t x = ent[i];
    const double* c = contrib + 9 * (int64_t)(x / 3) + 3 * (x % 3);
    g0 += c[0];
    g1 += c[1];
    g2 += c[2];
  }
  gv[3 * v + 0] = g0;
  gv[3 * v + 1] = g1;
  gv[3 * v + 2] = g2;
}

int64_t cdiv64(int64_t a, int64_t b) { return (a + b - 1) / b; }

int status_after_launch() { return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA; }

}  // namespace

// ---------------------------------------------------------------------------
// Plan and launchers (used by the C ABI in capi.cu).

constexpr int kR64 = 1, kF64 = 1;

Plan64 plan64(int64_t nv, int64_t nt, int64_t nfreq, const dm_box* box) {
  Plan64 p;
  CellDesc& d = p.d;
  memset(&d, 0, sizeof(d));
  for (int k = 0; k < 3; ++k) {
    d.lo[k] = box ? box->lo[k] : 0.0;
    d.len[k] = box ? box->hi[k] - box->lo[k] : 1.0;
    d.n[k] = box ? box->shape[k] : 1;
  }
  d.nv = (int32_t)nv;
  d.nt = (int32_t)nt;
  d.nband = (int32_t)nfreq;
  d.ne = d.nband;
  d.herm = 0;
  plan_cell_tiles_for(d, FwdVariant{kR64, kNT64, 8}, BwdVariant{kF64, kNT64, 8});
  p.face_blks = std::max<int64_t>(1, cdiv64(nt, kBlk64));
  p.band_blks = std::max<int64_t>(1, cdiv64(nfreq, kBlk64));
  p.fpart = (int64_t)d.fsplit * nfreq;
  p.bpart = (int64_t)d.bchunks * 10 * nt;
  p.fwd_items = (int64_t)d.xtiles * d.fsplit;
  p.bwd_items = (int64_t)d.fblocks * d.bchunks;
  return p;
}

size_t face64_bytes() { return sizeof(Face64); }
size_t xi64_bytes() { return sizeof(Xi64); }

int launch64_forward(const Plan64& p, const double* verts, const int64_t* faces,
                     const double* coeff, const int32_t* band_index, const double* xi_list,
                     const double* otf, void* recs, double* area_part, void* xrec, double* fpart,
                     double* ft_list, double* grid, int* err, cudaStream_t st) {
  const CellDesc& d = p.d;
  if (d.nt > 0)
    k64_face_prep<<<(unsigned)p.face_blks, kBlk64, 0, st>>>(d, verts, faces, coeff,
                                                           (Face64*)recs, area_part, err);
  else
    cudaMemsetAsync(area_part, 0, sizeof(double), st);
  if (d.nband <= 0) return status_after_launch();
  k64_xi_prep<<<(unsigned)p.band_blks, kBlk64, 0, st>>>(d, band_index, xi_list, nullptr, nullptr,
                                                       nullptr, 0.0, nullptr, (Xi64*)xrec,
                                                       nullptr, err);
  if (d.nt > 0) {
    k64_fwd<kR64><<<(unsigned)p.fwd_items, kNT64, 0, st>>>(d, (const Face64*)recs,
                                                          (const Xi64*)xrec, (double2*)fpart,
                                                          err);
  } else {
    cudaMemsetAsync(fpart, 0, sizeof(double2) * (size_t)std::max<int64_t>(p.fpart, 1), st);
  }
  k64_fwd_epi<<<(unsigned)p.band_blks, kBlk64, 0, st>>>(
      d, band_index, (const double2*)fpart, area_part, (int)(d.nt > 0 ? p.face_blks : 1), otf,
      (double2*)ft_list, (double2*)grid);
  count_launches(d.nt > 0 ? 4 : 2);
  return status_after_launch();
}

int launch64_backward(const Plan64& p, const double* verts, const int64_t* faces,
                      const double* coeff, const int32_t* band_index, const double* xi_list,
                      const double* grad_list, const double* grad_grid, const double* otf,
                      double grad_scale, const double* ft_list, const int32_t* csr_off,
                      const int32_t* csr_ent, void* recs, double* area_part, void* xrec,
                      double* s_part, double* bpart, double* contrib, double* grad_verts,
                      double* grad_coeff, int* err, cudaStream_t st) {
  const CellDesc& d = p.d;
  if (d.nt <= 0) {
    if (d.nv > 0) cudaMemsetAsync(grad_verts, 0, sizeof(double) * 3 * (size_t)d.nv, st);
    return status_after_launch();
  }
  k64_face_prep<<<(unsigned)p.face_blks, kBlk64, 0, st>>>(d, verts, faces, coeff, (Face64*)recs,
                                                         area_part, err);
  if (d.nband > 0) {
    k64_xi_prep<<<(unsigned)p.band_blks, kBlk64, 0, st>>>(
        d, band_index, xi_list, (const double2*)grad_list, (const double2*)grad_grid, otf,
        grad_scale, (const double2*)ft_list, (Xi64*)xrec, s_part, err);
    k64_bwd<kF64><<<(unsigned)p.bwd_items, kNT64, 0, st>>>(d, (const Face64*)recs,
                                                          (const Xi64*)xrec, bpart, err);
  } else {
    cudaMemsetAsync(s_part, 0, sizeof(double), st);
    cudaMemsetAsync(bpart, 0, sizeof(double) * (size_t)std::max<int64_t>(p.bpart, 1), st);
  }
  k64_face_epi<<<(unsigned)p.face_blks, kBlk64, 0, st>>>(
      d, (const Face64*)recs, coeff, area_part, (int)p.face_blks, s_part,
      (int)(d.nband > 0 ? p.band_blks : 1), bpart, contrib, grad_coeff);
  if (d.nv > 0)
    k64_vertex_gather<<<(unsigned)cdiv64(d.nv, kBlk64), kBlk64, 0, st>>>(d.nv, csr_off, csr_ent,
                                                                        contrib, grad_verts);
  count_launches(d.nband > 0 ? 5 : 3);
  return status_after_launch();
}

}  // namespace dm
