// Spatial PSF models of deltamic/psf.py on the GPU: the volume-sized stages.
//
//  * Anisotropic_gaussian_psf (psf.py:628-665): exp(-u^T S u / (2 D(z))) / D(z),
//    u = (x, y), D = eps + (|z| sigma_z)^2, and its gradient to (S, sigma_z, eps).
//  * Gibson_Lanni_psf (psf.py:23-154) is radially symmetric about the lateral
//    centre: its amplitude R(r) @ C depends on the pixel only through the pixel's
//    distance r from the centre.  The basis R(u, k) of psf.py:141-143 is formed
//    here for the distinct radii u only (a few thousand instead of nx*ny rows),
//    and the normalised intensity |A|^2 / max is scattered to the volume; the
//    backward gathers the volume gradient per radius.  The dense products
//    A = R C and its adjoints are plain cuBLAS GEMMs.
//  * Hanser_psf (psf.py:157-371): the pupil at every z plane,
//    P0 exp(2 pi i kz z) (psf.py:310-314, 336), and the intensity
//    |fftshift(field)|^2 permuted to (x, y, z) (psf.py:362, 264-266) around the
//    batched 2-D inverse FFT (cuFFT); Zernike polynomials (psf.py:373-548).
// Every reduction runs in a fixed order (block partials, then one final pass).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>

#include "../../include/deltamic_b200.h"
#include "dm_common.cuh"
#include "meshft_internal.h"

namespace dm {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 148 * 8;

int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }
int status() { return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA; }
unsigned grid_for(int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, kThreads), kMaxBlocks));
}

// Sum of kN doubles over the block into part[blockIdx.x * kN + i] (fixed order).
template <int kN>
__device__ void block_partials(double (&v)[kN], double* part) {
  __shared__ double sh[kN][kThreads / 32];
#pragma unroll
  for (int i = 0; i < kN; ++i) {
    double x = v[i];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sh[i][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < kN) {
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) s += sh[threadIdx.x][w];
    part[(int64_t)blockIdx.x * kN + threadIdx.x] = s;
  }
}

template <int kN, typename T>
__global__ void k_sum_partials(const double* __restrict__ part, int nblk, T* __restrict__ out) {
  if (threadIdx.x >= kN) return;
  double s = 0.0;
  for (int b = 0; b < nblk; ++b) s += part[(int64_t)b * kN + threadIdx.x];
  out[threadIdx.x] = (T)s;
}

// ---------------------------------------------------------------------------
// Anisotropic Gaussian

struct Grid3 {
  const float* x[3];
  int32_t n[3];
};

__device__ __forceinline__ void grid_point(int64_t i, const Grid3& g, float& x, float& y,
                                           float& z) {
  const int64_t n12 = (int64_t)g.n[1] * g.n[2];
  const int64_t a = i / n12;
  const int64_t r = i - a * n12;
  const int64_t b = r / g.n[2];
  x = g.x[0][a];
  y = g.x[1][b];
  z = g.x[2][r - b * g.n[2]];
}

// p = {s00, s01, s10, s11, sigma_z, eps}; float32 in the reference's operation order.
__global__ void k_aniso_psf(const float* __restrict__ p, Grid3 g, int64_t n,
                            float* __restrict__ out) {
  const float s00 = p[0], s01 = p[1], s10 = p[2], s11 = p[3], sz = p[4], eps = p[5];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float x, y, z;
    grid_point(i, g, x, y, z);
    const float q = x * (s00 * x + s01 * y) + y * (s10 * x + s11 * y);
    const float t = fabsf(z) * sz;
    const float D = eps + t * t;
    out[i] = expf(-q / (2.0f * D)) / D;
  }
}

// Per-block sums of g * d psf / d p_i for p = {s00, s01, s10, s11, sigma_z, eps}.
__global__ void k_aniso_psf_grad(const float* __restrict__ gpsf, const float* __restrict__ psf,
                                 const float* __restrict__ p, Grid3 g, int64_t n,
                                 double* __restrict__ part) {
  const double s00 = p[0], s01 = p[1], s10 = p[2], s11 = p[3], sz = p[4], eps = p[5];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float xf, yf, zf;
    grid_point(i, g, xf, yf, zf);
    const double x = xf, y = yf, z = zf;
    const double D = eps + (fabs(z) * sz) * (fabs(z) * sz);
    const double q = x * (s00 * x + s01 * y) + y * (s10 * x + s11 * y);
    const double ge = (double)gpsf[i] * (double)psf[i];
    const double w = -ge / (2.0 * D);  // d/d s_ij = w u_i u_j
    acc[0] += w * x * x;
    acc[1] += w * x * y;
    acc[2] += w * y * x;
    acc[3] += w * y * y;
    const double gD = ge * (q / (2.0 * D * D) - 1.0 / D);  // d/dD
    acc[4] += gD * 2.0 * z * z * sz;
    acc[5] += gD;
  }
  block_partials<6>(acc, part);
}

// ---------------------------------------------------------------------------
// Gibson-Lanni: radial basis and intensity

// R[u][k] = (s J1(s rm) J0(b rm) rm - b J0(s rm) J1(b rm) rm) / (s s - b b) with
// s = scaling[k], b = b[u], rm = *rhomax (psf.py:141-143), in the reference's
// operation order with every product and difference rounded on its own.  The
// Bessel values come in as tables, bs = {J0(s rm)}[K] ++ {J1(s rm)}[K] and
// bb = {J0(b rm)}[U] ++ {J1(b rm)}[U]: the amplitude R @ C cancels large terms of
// an ill-conditioned fit, so R must use the same Bessel values as the fit.
__device__ __forceinline__ void basis_terms(double s, double b, double rm, double J0s,
                                            double J1s, double J0b, double J1b, double& num,
                                            double& den) {
  num = __dsub_rn(__dmul_rn(__dmul_rn(__dmul_rn(s, J1s), J0b), rm),
                  __dmul_rn(__dmul_rn(__dmul_rn(b, J0s), J1b), rm));
  den = __dsub_rn(__dmul_rn(s, s), __dmul_rn(b, b));
}

__global__ void k_radial_basis(const double* __restrict__ scaling, int K,
                               const double* __restrict__ rhomax, const double* __restrict__ b,
                               int64_t U, const double* __restrict__ bs,
                               const double* __restrict__ bb, double* __restrict__ R) {
  const double rm = rhomax[0];
  const int64_t n = U * K;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t u = i / K;
    const int k = (int)(i - u * K);
    double num, den;
    basis_terms(scaling[k], b[u], rm, bs[k], bs[K + k], bb[u], bb[U + u], num, den);
    R[i] = __ddiv_rn(num, den);
  }
}

// J1(x)/x with its limit 1/2 at 0.
__device__ __forceinline__ double j1_over_x(double j1x, double x) {
  return fabs(x) < 1e-8 ? 0.5 - x * x / 16.0 : j1x / x;
}

// Partial derivatives of R(s, b, rm).  exact == 0: the Bessel values are
// constants, as in the reference (torch's bessel_j0 / bessel_j1 carry no
// gradient); exact != 0: also through them (J0' = -J1, J1'(x) = J0 - J1/x).
__device__ __forceinline__ void basis_partials(double s, double b, double rm, double J0s,
                                               double J1s, double J0b, double J1b, int exact,
                                               double& ds, double& db, double& dr) {
  const double num = s * J1s * J0b * rm - b * J0s * J1b * rm;
  const double den = s * s - b * b;
  double dns = J1s * J0b * rm, dnb = -J0s * J1b * rm, dnr = s * J1s * J0b - b * J0s * J1b;
  if (exact) {
    const double a = s * rm, c = b * rm;
    const double dJ1s = J0s - j1_over_x(J1s, a), dJ1b = J0b - j1_over_x(J1b, c);
    dns += s * dJ1s * rm * J0b * rm + b * J1s * rm * J1b * rm;
    dnb += -s * J1s * J1b * rm * rm - b * J0s * dJ1b * rm * rm;
    dnr += s * s * dJ1s * J0b * rm - s * b * J1s * J1b * rm + b * s * J1s * J1b * rm -
           b * b * J0s * dJ1b * rm;
  }
  ds = (dns * den - num * 2.0 * s) / (den * den);
  db = (dnb * den + num * 2.0 * b) / (den * den);
  dr = dnr / den;
}

// gb[u] = sum_k gR dR/db, ds[u][k] = gR dR/ds, and per-block sums of gR dR/d rm
// (u in blocks, k in order).
__global__ void k_radial_basis_grad_u(const double* __restrict__ gR,
                                      const double* __restrict__ scaling, int K,
                                      const double* __restrict__ rhomax,
                                      const double* __restrict__ b, int64_t U,
                                      const double* __restrict__ bs,
                                      const double* __restrict__ bb, int exact,
                                      double* __restrict__ gb, double* __restrict__ ds_out,
                                      double* __restrict__ part) {
  const double rm = rhomax[0];
  const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  if (u < U) {
    double sb = 0.0;
    for (int k = 0; k < K; ++k) {
      double ds, db, dr;
      basis_partials(scaling[k], b[u], rm, bs[k], bs[K + k], bb[u], bb[U + u], exact, ds, db,
                     dr);
      const double g = gR[u * K + k];
      sb += g * db;
      acc[0] += g * dr;
      ds_out[u * K + k] = g * ds;
    }
    gb[u] = sb;
  }
  block_partials<1>(acc, part);
}

// gscaling[k] = sum_u ds[u][k]: one block per k, a fixed-order tree over u.
__global__ void k_radial_basis_grad_k(const double* __restrict__ ds, int K, int64_t U,
                                      double* __restrict__ gscaling) {
  __shared__ double sh[kThreads / 32];
  const int k = blockIdx.x;
  double x = 0.0;
  for (int64_t u = threadIdx.x; u < U; u += blockDim.x) x += ds[u * K + k];
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) t += sh[w];
    gscaling[k] = t;
  }
}

// prof[u][z] = |A[u][z]|^2 and per-block maxima.
__global__ void k_radial_intensity(const double2* __restrict__ A, int64_t n,
                                   double* __restrict__ prof, double* __restrict__ part) {
  double mx = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 a = A[i];
    const double p = a.x * a.x + a.y * a.y;
    prof[i] = p;
    mx = fmax(mx, p);
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  __shared__ double sh[kThreads / 32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) m = fmax(m, sh[w]);
    part[blockIdx.x] = m;
  }
}

__global__ void k_max_final(const double* __restrict__ part, int nblk, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double m = 0.0;
  for (int b = 0; b < nblk; ++b) m = fmax(m, part[b]);
  out[0] = m;
}

// psf[p][z] = prof[pix[p]][z] / peak (z fastest: coalesced reads and writes).
__global__ void k_radial_scatter(const double* __restrict__ prof, const int32_t* __restrict__ pix,
                                 int64_t npix, int nz, const double* __restrict__ peak,
                                 double* __restrict__ psf) {
  const double inv = 1.0 / peak[0];
  const int64_t n = npix * nz;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / nz;
    const int z = (int)(i - p * nz);
    psf[i] = prof[(int64_t)pix[p] * nz + z] * inv;
  }
}

// S[u][z] = sum of g over the pixels of radius u (CSR, in order); per-block sums
// of S * prof and of the pixels tied with the peak.
__global__ void k_radial_gather(const double* __restrict__ g, const int32_t* __restrict__ off,
                                const int32_t* __restrict__ pixels, int64_t U, int nz,
                                const double* __restrict__ prof, const double* __restrict__ peak,
                                double* __restrict__ S, double* __restrict__ part) {
  const double m = peak[0];
  double acc[2] = {0.0, 0.0};
  const int64_t n = U * nz;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t u = i / nz;
    const int z = (int)(i - u * nz);
    double s = 0.0;
    for (int32_t e = off[u]; e < off[u + 1]; ++e) s += g[(int64_t)pixels[e] * nz + z];
    S[i] = s;
    acc[0] += s * prof[i];
    if (prof[i] == m) acc[1] += (double)(off[u + 1] - off[u]);
  }
  block_partials<2>(acc, part);
}

// gA[u][z] = 2 A (S/m - [prof == m] cnt(u) GS / (m^2 ties)): the adjoint of
// psf = prof / max(prof) with the max's gradient shared by its ties (torch).
__global__ void k_radial_grad_amp(const double2* __restrict__ A, const double* __restrict__ S,
                                  const double* __restrict__ prof,
                                  const int32_t* __restrict__ off, int64_t U, int nz,
                                  const double* __restrict__ peak,
                                  const double* __restrict__ sums, double2* __restrict__ gA) {
  const double m = peak[0], GS = sums[0], ties = sums[1];
  const int64_t n = U * nz;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t u = i / nz;
    double gp = S[i] / m;
    if (prof[i] == m) gp -= (double)(off[u + 1] - off[u]) * GS / (m * m * ties);
    const double2 a = A[i];
    gA[i] = make_double2(2.0 * gp * a.x, 2.0 * gp * a.y);
  }
}

// ---------------------------------------------------------------------------
// Hanser: pupil planes, shifted intensity, Zernike polynomials

constexpr float kTwoPiF = 6.28318530717958647692f;

// pupil[z][x][y] = P0[x][y] exp(2 pi i kz[x][y] zr[z]).
__global__ void k_pupil_defocus(const float2* __restrict__ P0, const float* __restrict__ kz,
                                const float* __restrict__ zr, int64_t nxy, int nz,
                                float2* __restrict__ pupil) {
  const int64_t n = nxy * nz;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t z = i / nxy;
    const int64_t p = i - z * nxy;
    float s, c;
    sincosf(kTwoPiF * kz[p] * zr[z], &s, &c);
    const float2 a = P0[p];
    pupil[i] = make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
  }
}

// Backward of k_pupil_defocus for cotangent gp[z][x][y]: per (x, y)
//   gP0 = sum_z gp conj(e),  gkz = sum_z Re(conj(gp) 2 pi i zr P0 e),
// and per-block partial sums over (x, y) of gzr[z] = Re(conj(gp) 2 pi i kz P0 e).
__global__ void k_pupil_defocus_grad(const float2* __restrict__ gp, const float2* __restrict__ P0,
                                     const float* __restrict__ kz, const float* __restrict__ zr,
                                     int64_t nxy, int nz, float2* __restrict__ gP0,
                                     float* __restrict__ gkz, double* __restrict__ part) {
  __shared__ double sh[kThreads / 32];
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = p < nxy;
  const float2 a = live ? P0[p] : make_float2(0.f, 0.f);
  const float k = live ? kz[p] : 0.f;
  double sx = 0.0, sy = 0.0, sk = 0.0;
  for (int z = 0; z < nz; ++z) {
    double tz = 0.0;
    if (live) {
      float s, c;
      sincosf(kTwoPiF * k * zr[z], &s, &c);
      const float2 g = gp[(int64_t)z * nxy + p];
      // conj(e) g
      sx += (double)(c * g.x + s * g.y);
      sy += (double)(c * g.y - s * g.x);
      // v = P0 e; Re(conj(g) i v) = g.x (-v.y) + g.y v.x
      const float vx = a.x * c - a.y * s, vy = a.x * s + a.y * c;
      const double re = (double)g.y * vx - (double)g.x * vy;
      sk += re * (double)kTwoPiF * zr[z];
      tz = re * (double)kTwoPiF * k;
    }
    for (int o = 16; o > 0; o >>= 1) tz += __shfl_down_sync(0xffffffffu, tz, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = tz;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kThreads / 32; ++w) t += sh[w];
      part[(int64_t)blockIdx.x * nz + z] = t;
    }
    __syncthreads();
  }
  if (live) {
    gP0[p] = make_float2((float)sx, (float)sy);
    gkz[p] = (float)sk;
  }
}

__global__ void k_sum_columns(const double* __restrict__ part, int nblk, int nz,
                              float* __restrict__ out) {
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= nz) return;
  double s = 0.0;
  for (int b = 0; b < nblk; ++b) s += part[(int64_t)b * nz + z];
  out[z] = (float)s;
}

// out[x][y][z] = |field[z][(x - nx/2) mod nx][(y - ny/2) mod ny]|^2 (fftshift over
// x, y, then (z, x, y) -> (x, y, z)); a 32 x 32 (y, z) tile per block through
// shared memory so both sides are coalesced.  With kBack the adjoint:
// gfield[z][x'][y'] = 2 gout[x][y][z] field[z][x'][y'].
template <bool kBack>
__global__ void k_shifted_intensity(const float2* __restrict__ field,
                                    const float* __restrict__ gout, int nx, int ny, int nz,
                                    float* __restrict__ out, float2* __restrict__ gfield) {
  __shared__ float tile[32][33];
  const int x = blockIdx.z;
  const int y0 = blockIdx.x * 32, z0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  const int xs = (x - nx / 2 + nx) % nx;
  if (!kBack) {
    for (int j = ty; j < 32; j += 8) {  // read: z = z0 + j, y = y0 + tx
      const int z = z0 + j, y = y0 + tx;
      float v = 0.f;
      if (z < nz && y < ny) {
        const int ys = (y - ny / 2 + ny) % ny;
        const float2 f = field[((int64_t)z * nx + xs) * ny + ys];
        v = f.x * f.x + f.y * f.y;
      }
      tile[j][tx] = v;
    }
    __syncthreads();
    for (int j = ty; j < 32; j += 8) {  // write: y = y0 + j, z = z0 + tx
      const int y = y0 + j, z = z0 + tx;
      if (y < ny && z < nz) out[((int64_t)x * ny + y) * nz + z] = tile[tx][j];
    }
  } else {
    for (int j = ty; j < 32; j += 8) {  // read gout: y = y0 + j, z = z0 + tx
      const int y = y0 + j, z = z0 + tx;
      tile[j][tx] = (y < ny && z < nz) ? gout[((int64_t)x * ny + y) * nz + z] : 0.f;
    }
    __syncthreads();
    for (int j = ty; j < 32; j += 8) {  // write gfield: z = z0 + j, y = y0 + tx
      const int z = z0 + j, y = y0 + tx;
      if (z < nz && y < ny) {
        const int ys = (y - ny / 2 + ny) % ny;
        const int64_t o = ((int64_t)z * nx + xs) * ny + ys;
        const float2 f = field[o];
        const float g = 2.0f * tile[tx][j];
        gfield[o] = make_float2(g * f.x, g * f.y);
      }
    }
  }
}

constexpr int kZernMaxModes = 66;  // radial degree up to 10
constexpr int kZernMaxTerms = 6;
struct ZernTable {
  int32_t n_modes;
  int32_t m[kZernMaxModes];        // signed azimuthal degree
  int32_t terms[kZernMaxModes];    // terms of the radial polynomial in r^2
  double norm[kZernMaxModes];
  double c[kZernMaxModes][kZernMaxTerms];  // R = r^|m| sum_t c[t] (r^2)^t
};

// out[j][i] = Z_j(r[i], theta[i]) (0 outside the unit disk), float64 arithmetic.
__global__ void k_zernike(const float* __restrict__ r, const float* __restrict__ theta,
                          int64_t n, ZernTable t, float* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double rr = r[i], th = theta[i];
    const bool in = rr <= 1.0;
    const double q = rr * rr;
    for (int j = 0; j < t.n_modes; ++j) {
      double v = 0.0;
      if (in) {
        const int am = abs(t.m[j]);
        double poly = 0.0;
        for (int k = t.terms[j] - 1; k >= 0; --k) poly = poly * q + t.c[j][k];
        double rm = 1.0;
        for (int e = 0; e < am; ++e) rm *= rr;
        const double ang = t.m[j] < 0 ? sin(am * th) : cos(am * th);
        v = rm * poly * ang * t.norm[j];
      }
      out[(int64_t)j * n + i] = (float)v;
    }
  }
}

double factorial(int n) {
  double f = 1.0;
  for (int i = 2; i <= n; ++i) f *= i;
  return f;
}

}  // namespace
}  // namespace dm

using namespace dm;

extern "C" {

int dm_aniso_gaussian_psf(const float* params, const float* x, int32_t nx, const float* y,
                          int32_t ny, const float* z, int32_t nz, float* psf,
                          dm_stream_t stream) {
  if (!params || !x || !y || !z || !psf || nx <= 0 || ny <= 0 || nz <= 0)
    return DM_ERR_INVALID_ARG;
  const int64_t n = (int64_t)nx * ny * nz;
  Grid3 g{{x, y, z}, {nx, ny, nz}};
  k_aniso_psf<<<grid_for(n), kThreads, 0, (cudaStream_t)stream>>>(params, g, n, psf);
  count_launches(1);
  return status();
}

size_t dm_aniso_gaussian_psf_grad_workspace_size(int64_t n) {
  if (n < 0) return 0;
  return sizeof(double) * 6 * (size_t)grid_for(n) + 256;
}

int dm_aniso_gaussian_psf_grad(const float* grad_psf, const float* psf, const float* params,
                               const float* x, int32_t nx, const float* y, int32_t ny,
                               const float* z, int32_t nz, float* grad_params, void* workspace,
                               size_t ws_bytes, dm_stream_t stream) {
  if (!grad_psf || !psf || !params || !x || !y || !z || !grad_params || !workspace ||
      nx <= 0 || ny <= 0 || nz <= 0)
    return DM_ERR_INVALID_ARG;
  const int64_t n = (int64_t)nx * ny * nz;
  if (ws_bytes < dm_aniso_gaussian_psf_grad_workspace_size(n)) return DM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned nb = grid_for(n);
  Grid3 g{{x, y, z}, {nx, ny, nz}};
  double* part = (double*)workspace;
  k_aniso_psf_grad<<<nb, kThreads, 0, st>>>(grad_psf, psf, params, g, n, part);
  k_sum_partials<6, float><<<1, 32, 0, st>>>(part, (int)nb, grad_params);
  count_launches(2);
  return status();
}

int dm_radial_basis(const double* scaling, int32_t n_basis, const double* rhomax,
                    const double* b, int64_t n_radii, const double* bessel_s,
                    const double* bessel_b, double* basis, dm_stream_t stream) {
  if (!scaling || !rhomax || !b || !bessel_s || !bessel_b || !basis || n_basis <= 0 ||
      n_radii <= 0)
    return DM_ERR_INVALID_ARG;
  const int64_t n = n_radii * n_basis;
  k_radial_basis<<<grid_for(n), kThreads, 0, (cudaStream_t)stream>>>(
      scaling, n_basis, rhomax, b, n_radii, bessel_s, bessel_b, basis);
  count_launches(1);
  return status();
}

size_t dm_radial_basis_grad_workspace_size(int64_t n_radii, int32_t n_basis) {
  if (n_radii <= 0 || n_basis <= 0) return 0;
  return sizeof(double) * ((size_t)cdiv(n_radii, kThreads) + (size_t)n_radii * n_basis) + 512;
}

int dm_radial_basis_grad(const double* grad_basis, const double* scaling, int32_t n_basis,
                         const double* rhomax, const double* b, int64_t n_radii,
                         const double* bessel_s, const double* bessel_b, int32_t exact,
                         double* grad_scaling, double* grad_rhomax, double* grad_b,
                         void* workspace, size_t ws_bytes, dm_stream_t stream) {
  if (!grad_basis || !scaling || !rhomax || !b || !bessel_s || !bessel_b || !grad_scaling ||
      !grad_rhomax || !grad_b || !workspace || n_basis <= 0 || n_radii <= 0)
    return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm_radial_basis_grad_workspace_size(n_radii, n_basis)) return DM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned nb = (unsigned)cdiv(n_radii, kThreads);
  double* part = (double*)workspace;
  double* ds = part + nb;
  k_radial_basis_grad_u<<<nb, kThreads, 0, st>>>(grad_basis, scaling, n_basis, rhomax, b,
                                                n_radii, bessel_s, bessel_b, exact, grad_b, ds,
                                                part);
  k_radial_basis_grad_k<<<(unsigned)n_basis, kThreads, 0, st>>>(ds, n_basis, n_radii,
                                                                grad_scaling);
  k_sum_partials<1, double><<<1, 32, 0, st>>>(part, (int)nb, grad_rhomax);
  count_launches(3);
  return status();
}

size_t dm_radial_intensity_workspace_size(int64_t n_radii, int32_t nz) {
  if (n_radii <= 0 || nz <= 0) return 0;
  const int64_t n = n_radii * nz;
  return sizeof(double) * (2 * (size_t)n + 2 * (size_t)grid_for(n) + 4) + 512;
}

int dm_radial_intensity(const double* amp, int64_t n_radii, int32_t nz, const int32_t* pixel_radius,
                        int64_t n_pixels, double* psf, double* profile, double* peak,
                        void* workspace, size_t ws_bytes, dm_stream_t stream) {
  if (!amp || !pixel_radius || !psf || !profile || !peak || !workspace || n_radii <= 0 ||
      nz <= 0 || n_pixels <= 0)
    return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm_radial_intensity_workspace_size(n_radii, nz)) return DM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n = n_radii * nz;
  const unsigned nb = grid_for(n);
  double* part = (double*)workspace;
  k_radial_intensity<<<nb, kThreads, 0, st>>>((const double2*)amp, n, profile, part);
  k_max_final<<<1, 32, 0, st>>>(part, (int)nb, peak);
  k_radial_scatter<<<grid_for(n_pixels * nz), kThreads, 0, st>>>(profile, pixel_radius,
                                                                 n_pixels, nz, peak, psf);
  count_launches(3);
  return status();
}

int dm_radial_intensity_backward(const double* grad_psf, const double* amp, const double* profile,
                                 const double* peak, int64_t n_radii, int32_t nz,
                                 const int32_t* radius_off, const int32_t* radius_pixels,
                                 double* grad_amp, void* workspace, size_t ws_bytes,
                                 dm_stream_t stream) {
  if (!grad_psf || !amp || !profile || !peak || !radius_off || !radius_pixels || !grad_amp ||
      !workspace || n_radii <= 0 || nz <= 0)
    return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm_radial_intensity_workspace_size(n_radii, nz)) return DM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n = n_radii * nz;
  const unsigned nb = grid_for(n);
  double* S = (double*)workspace;
  double* part = S + n;
  double* sums = part + 2 * (size_t)nb;
  k_radial_gather<<<nb, kThreads, 0, st>>>(grad_psf, radius_off, radius_pixels, n_radii, nz,
                                          profile, peak, S, part);
  k_sum_partials<2, double><<<1, 32, 0, st>>>(part, (int)nb, sums);
  k_radial_grad_amp<<<nb, kThreads, 0, st>>>((const double2*)amp, S, profile, radius_off,
                                            n_radii, nz, peak, sums, (double2*)grad_amp);
  count_launches(3);
  return status();
}

int dm_pupil_defocus(const float* pupil0, const float* kz, const float* zr, int32_t nx,
                     int32_t ny, int32_t nz, float* pupil, dm_stream_t stream) {
  if (!pupil0 || !kz || !zr || !pupil || nx <= 0 || ny <= 0 || nz <= 0)
    return DM_ERR_INVALID_ARG;
  const int64_t nxy = (int64_t)nx * ny;
  k_pupil_defocus<<<grid_for(nxy * nz), kThreads, 0, (cudaStream_t)stream>>>(
      (const float2*)pupil0, kz, zr, nxy, nz, (float2*)pupil);
  count_launches(1);
  return status();
}

size_t dm_pupil_defocus_grad_workspace_size(int32_t nx, int32_t ny, int32_t nz) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return 0;
  return sizeof(double) * (size_t)cdiv((int64_t)nx * ny, kThreads) * (size_t)nz + 256;
}

int dm_pupil_defocus_backward(const float* grad_pupil, const float* pupil0, const float* kz,
                              const float* zr, int32_t nx, int32_t ny, int32_t nz,
                              float* grad_pupil0, float* grad_kz, float* grad_zr,
                              void* workspace, size_t ws_bytes, dm_stream_t stream) {
  if (!grad_pupil || !pupil0 || !kz || !zr || !grad_pupil0 || !grad_kz || !grad_zr ||
      !workspace || nx <= 0 || ny <= 0 || nz <= 0)
    return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm_pupil_defocus_grad_workspace_size(nx, ny, nz)) return DM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t nxy = (int64_t)nx * ny;
  const int nb = (int)cdiv(nxy, kThreads);
  double* part = (double*)workspace;
  k_pupil_defocus_grad<<<nb, kThreads, 0, st>>>((const float2*)grad_pupil, (const float2*)pupil0,
                                               kz, zr, nxy, nz, (float2*)grad_pupil0, grad_kz,
                                               part);
  k_sum_columns<<<(unsigned)cdiv(nz, 128), 128, 0, st>>>(part, nb, nz, grad_zr);
  count_launches(2);
  return status();
}

int dm_shifted_intensity(const float* field, int32_t nx, int32_t ny, int32_t nz, float* out,
                         dm_stream_t stream) {
  if (!field || !out || nx <= 0 || ny <= 0 || nz <= 0) return DM_ERR_INVALID_ARG;
  if (nx > 65535) return DM_ERR_SIZE;
  const dim3 grid((unsigned)cdiv(ny, 32), (unsigned)cdiv(nz, 32), (unsigned)nx);
  k_shifted_intensity<false><<<grid, 256, 0, (cudaStream_t)stream>>>(
      (const float2*)field, nullptr, nx, ny, nz, out, nullptr);
  count_launches(1);
  return status();
}

int dm_shifted_intensity_backward(const float* field, const float* grad_out, int32_t nx,
                                  int32_t ny, int32_t nz, float* grad_field, dm_stream_t stream) {
  if (!field || !grad_out || !grad_field || nx <= 0 || ny <= 0 || nz <= 0)
    return DM_ERR_INVALID_ARG;
  if (nx > 65535) return DM_ERR_SIZE;
  const dim3 grid((unsigned)cdiv(ny, 32), (unsigned)cdiv(nz, 32), (unsigned)nx);
  k_shifted_intensity<true><<<grid, 256, 0, (cudaStream_t)stream>>>(
      (const float2*)field, grad_out, nx, ny, nz, nullptr, (float2*)grad_field);
  count_launches(1);
  return status();
}

int dm_zernike(const float* r, const float* theta, int64_t n_points, const int32_t* degrees,
               int32_t n_modes, float* out, dm_stream_t stream) {
  if (!r || !theta || !degrees || !out || n_points < 0 || n_modes <= 0 ||
      n_modes > kZernMaxModes)
    return DM_ERR_INVALID_ARG;
  ZernTable t;
  memset(&t, 0, sizeof(t));
  t.n_modes = n_modes;
  for (int j = 0; j < n_modes; ++j) {
    const int n = degrees[2 * j], m = degrees[2 * j + 1], am = abs(m);
    if (n < 0 || am > n || n > 10) return DM_ERR_INVALID_ARG;
    t.m[j] = m;
    t.norm[j] = m == 0 ? sqrt((double)(n + 1)) : sqrt(2.0 * (n + 1));
    if ((n - am) % 2) {  // not a Zernike polynomial: zero (psf.py:527-528)
      t.terms[j] = 0;
      continue;
    }
    const int h = (n - am) / 2;
    t.terms[j] = h + 1;
    // R = sum_s (-1)^s (n-s)! / (s! ((n+m)/2-s)! ((n-m)/2-s)!) r^(n-2s); in powers of
    // r^2 after r^|m|: the term s goes to power h - s.
    for (int s = 0; s <= h; ++s) {
      const double c = ((s % 2) ? -1.0 : 1.0) * factorial(n - s) /
                       (factorial(s) * factorial((n + am) / 2 - s) * factorial(h - s));
      t.c[j][h - s] = c;
    }
  }
  if (n_points == 0) return DM_OK;
  k_zernike<<<grid_for(n_points), kThreads, 0, (cudaStream_t)stream>>>(r, theta, n_points, t,
                                                                        out);
  count_launches(1);
  return status();
}

}  // extern "C"
