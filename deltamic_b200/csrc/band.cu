// Narrow-band compaction and the Gaussian OTF (forward and sigma gradient).
//
// Both are HBM-bound streams over the n0*n1*n2 grid: compaction reads the OTF
// twice (count, then write) and writes 4 bytes per band voxel; the OTF kernel
// writes 4 bytes per voxel; the sigma gradient reads 8 bytes per voxel.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "band_internal.h"
#include "dm_common.cuh"

namespace dm {

constexpr int kBandThreads = 256;
constexpr int kBandPerThread = 16;
constexpr int kBandTile = kBandThreads * kBandPerThread;  // voxels per block

// Per-block count of otf > thresh over contiguous tiles (float or double OTF).
template <typename T>
__global__ void k_band_count(const T* __restrict__ otf, int64_t n, T thresh,
                             int32_t* __restrict__ blk_count) {
  __shared__ int32_t sh[kBandThreads / 32];
  const int64_t base = (int64_t)blockIdx.x * kBandTile;
  int32_t c = 0;
#pragma unroll
  for (int k = 0; k < kBandPerThread; ++k) {
    const int64_t i = base + (int64_t)k * kBandThreads + threadIdx.x;
    if (i < n && otf[i] > thresh) ++c;
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int32_t s = 0;
    for (int w = 0; w < kBandThreads / 32; ++w) s += sh[w];
    blk_count[blockIdx.x] = s;
  }
}

// Exclusive scan of the block counts (one block); total to *count.
__global__ void k_band_scan(const int32_t* __restrict__ blk_count, int32_t* __restrict__ blk_off,
                            int64_t nblk, int64_t* __restrict__ count) {
  __shared__ int64_t sh[1024];
  const int T = blockDim.x;
  const int64_t per = (nblk + T - 1) / T;
  const int64_t b = threadIdx.x * per;
  const int64_t e = (b + per < nblk) ? b + per : nblk;
  int64_t s = 0;
  for (int64_t i = b; i < e; ++i) s += blk_count[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < T; o <<= 1) {
    const int64_t v = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += v;
    __syncthreads();
  }
  int64_t run = sh[threadIdx.x] - s;
  for (int64_t i = b; i < e; ++i) {
    blk_off[i] = (int32_t)run;
    run += blk_count[i];
  }
  if (threadIdx.x == T - 1) *count = sh[T - 1];
}

// Write the indices in ascending order: within a block, tile k of the block is
// handled in order and each warp-level ballot gives the rank inside the tile.
template <typename T>
__global__ void k_band_write(const T* __restrict__ otf, int64_t n, T thresh,
                             const int32_t* __restrict__ blk_off, int32_t* __restrict__ out) {
  __shared__ int32_t wsum[kBandThreads / 32];
  __shared__ int32_t run;
  const int64_t base = (int64_t)blockIdx.x * kBandTile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) run = blk_off[blockIdx.x];
  __syncthreads();
  for (int k = 0; k < kBandPerThread; ++k) {
    const int64_t i = base + (int64_t)k * kBandThreads + threadIdx.x;
    const bool p = i < n && otf[i] > thresh;
    const uint32_t bal = __ballot_sync(0xffffffffu, p);
    if (lane == 0) wsum[warp] = __popc(bal);
    __syncthreads();
    int32_t before = run;
    for (int w = 0; w < warp; ++w) before += wsum[w];
    if (p) out[before + __popc(bal & ((1u << lane) - 1u))] = (int32_t)i;
    __syncthreads();
    if (threadIdx.x == 0) {
      int32_t t = 0;
      for (int w = 0; w < kBandThreads / 32; ++w) t += wsum[w];
      run += t;
    }
    __syncthreads();
  }
}

int64_t band_blocks(int64_t n) { return (n + kBandTile - 1) / kBandTile; }

template <typename T>
static int launch_narrowband_t(const T* otf, int64_t n, T thresh, int32_t* out, int64_t* count,
                               int32_t* blk_count, int32_t* blk_off, cudaStream_t st) {
  const int64_t nb = band_blocks(n);
  if (nb > 0) {
    k_band_count<T><<<(unsigned)nb, kBandThreads, 0, st>>>(otf, n, thresh, blk_count);
  }
  k_band_scan<<<1, 1024, 0, st>>>(blk_count, blk_off, nb, count);
  if (nb > 0)
    k_band_write<T><<<(unsigned)nb, kBandThreads, 0, st>>>(otf, n, thresh, blk_off, out);
  count_launches(1 + (nb > 0 ? 2 : 0));
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

int launch_narrowband(const float* otf, int64_t n, float thresh, int32_t* out, int64_t* count,
                      int32_t* blk_count, int32_t* blk_off, cudaStream_t st) {
  return launch_narrowband_t<float>(otf, n, thresh, out, count, blk_count, blk_off, st);
}

int launch_narrowband64(const double* otf, int64_t n, double thresh, int32_t* out,
                        int64_t* count, int32_t* blk_count, int32_t* blk_off, cudaStream_t st) {
  return launch_narrowband_t<double>(otf, n, thresh, out, count, blk_count, blk_off, st);
}

// Mirror test of a band (DM_BAND_HERMITIAN): one block, fixed result.
__global__ void k_band_mirror(const int32_t* __restrict__ band, int64_t nb, int64_t nvox,
                              int32_t* __restrict__ flag) {
  int ok = 1;
  for (int64_t m = threadIdx.x; m < nb; m += blockDim.x)
    ok &= (int64_t)band[nb - 1 - m] == nvox - 1 - (int64_t)band[m];
  ok = __syncthreads_and(ok);
  if (threadIdx.x == 0) *flag = ok;
}

int launch_band_mirror(const int32_t* band, int64_t nb, int64_t nvox, int32_t* flag,
                       cudaStream_t st) {
  k_band_mirror<<<1, 1024, 0, st>>>(band, nb, nvox, flag);
  count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// Gaussian OTF exp(-(xi^T S xi)/2) (generate_gaussian_psf, psf.py:15-20) on the
// outer grid of three frequency axes, with the float32 operation order of the
// reference expression (no contraction into FMAs).

template <typename T>
struct AxesT {
  const T* x[3];
  int32_t n[3];
};

template <typename T>
__device__ __forceinline__ void grid_xi(int64_t i, const AxesT<T>& a, T x[3]) {
  const int64_t n12 = (int64_t)a.n[1] * a.n[2];
  const int32_t k0 = (int32_t)(i / n12);
  const int64_t rem = i - (int64_t)k0 * n12;
  const int32_t k1 = (int32_t)(rem / a.n[2]);
  const int32_t k2 = (int32_t)(rem - (int64_t)k1 * a.n[2]);
  x[0] = a.x[0][k0];
  x[1] = a.x[1][k1];
  x[2] = a.x[2][k2];
}

// Rounded products and sums in the reference expression's order (no FMA).
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float expT(float x) { return expf(x); }
__device__ __forceinline__ double expT(double x) { return exp(x); }

template <typename T>
__device__ __forceinline__ T quad_form(const T S[9], const T x[3]) {
  T q = 0;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    T t = radd(rmul(S[3 * r + 0], x[0]), rmul(S[3 * r + 1], x[1]));
    t = radd(t, rmul(S[3 * r + 2], x[2]));
    const T p = rmul(x[r], t);
    q = r == 0 ? p : radd(q, p);
  }
  return q;
}

template <typename T>
__global__ void k_gaussian_otf(const T* __restrict__ sigma, AxesT<T> a, int64_t n,
                               T* __restrict__ otf) {
  T S[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) S[k] = sigma[k];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    T x[3];
    grid_xi(i, a, x);
    otf[i] = expT(-quad_form(S, x) / (T)2);
  }
}

// Partial sums of grad_otf * otf * (-x_i x_j / 2) for the 6 distinct (i <= j).
template <typename T>
__global__ void k_otf_sigma_grad_part(const T* __restrict__ gotf,
                                      const int32_t* __restrict__ band, int64_t n,
                                      const T* __restrict__ otf, AxesT<T> a,
                                      double* __restrict__ part) {
  const int64_t nvox = (int64_t)a.n[0] * a.n[1] * a.n[2];
  __shared__ double sh[6][kBandThreads / 32];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = band ? (int64_t)band[i] : i;
    if (v < 0 || v >= nvox) continue;  // indices outside the grid contribute nothing
    T xt[3];
    grid_xi(v, a, xt);
    const double x[3] = {(double)xt[0], (double)xt[1], (double)xt[2]};
    const double w = -0.5 * (double)gotf[i] * (double)otf[v];
    acc[0] += w * x[0] * x[0];
    acc[1] += w * x[0] * x[1];
    acc[2] += w * x[0] * x[2];
    acc[3] += w * x[1] * x[1];
    acc[4] += w * x[1] * x[2];
    acc[5] += w * x[2] * x[2];
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double s = 0.0;
    for (int w = 0; w < kBandThreads / 32; ++w) s += sh[threadIdx.x][w];
    part[6 * blockIdx.x + threadIdx.x] = s;
  }
}

template <typename T>
__global__ void k_otf_sigma_grad_final(const double* __restrict__ part, int nblk,
                                       T* __restrict__ grad_sigma) {
  if (threadIdx.x >= 6) return;
  double s = 0.0;
  for (int b = 0; b < nblk; ++b) s += part[6 * b + threadIdx.x];
  const int ij[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  const int i = ij[threadIdx.x][0], j = ij[threadIdx.x][1];
  grad_sigma[3 * i + j] = (T)s;
  grad_sigma[3 * j + i] = (T)s;
}

template <typename T>
static AxesT<T> make_axes(const T* const xi[3], const int32_t n[3]) {
  AxesT<T> a;
  for (int d = 0; d < 3; ++d) {
    a.x[d] = xi[d];
    a.n[d] = n[d];
  }
  return a;
}

template <typename T>
static int launch_gaussian_otf_t(const T* sigma, const T* const xi[3], const int32_t n[3],
                                 T* otf, cudaStream_t st) {
  const int64_t nv = (int64_t)n[0] * n[1] * n[2];
  const int64_t blocks = std::min<int64_t>((nv + 255) / 256, 148 * 32);
  if (nv > 0) {
    k_gaussian_otf<T><<<(unsigned)blocks, 256, 0, st>>>(sigma, make_axes<T>(xi, n), nv, otf);
    count_launches(1);
  }
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

int launch_gaussian_otf(const float* sigma, const float* const xi[3], const int32_t n[3],
                        float* otf, cudaStream_t st) {
  return launch_gaussian_otf_t<float>(sigma, xi, n, otf, st);
}

int launch_gaussian_otf64(const double* sigma, const double* const xi[3], const int32_t n[3],
                          double* otf, cudaStream_t st) {
  return launch_gaussian_otf_t<double>(sigma, xi, n, otf, st);
}

int otf_grad_blocks(int64_t n) {
  const int64_t b = (n + kBandThreads - 1) / kBandThreads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 8));
}

template <typename T>
static int launch_otf_sigma_grad_t(const T* gotf, const int32_t* band, int64_t n, const T* otf,
                                   const T* const xi[3], const int32_t nax[3], T* grad_sigma,
                                   double* part, cudaStream_t st) {
  const int nblk = otf_grad_blocks(n);
  k_otf_sigma_grad_part<T><<<nblk, kBandThreads, 0, st>>>(gotf, band, n, otf,
                                                          make_axes<T>(xi, nax), part);
  k_otf_sigma_grad_final<T><<<1, 32, 0, st>>>(part, nblk, grad_sigma);
  count_launches(2);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

int launch_otf_sigma_grad(const float* gotf, const int32_t* band, int64_t n, const float* otf,
                          const float* const xi[3], const int32_t nax[3], float* grad_sigma,
                          double* part, cudaStream_t st) {
  return launch_otf_sigma_grad_t<float>(gotf, band, n, otf, xi, nax, grad_sigma, part, st);
}

int launch_otf_sigma_grad64(const double* gotf, const int32_t* band, int64_t n,
                            const double* otf, const double* const xi[3], const int32_t nax[3],
                            double* grad_sigma, double* part, cudaStream_t st) {
  return launch_otf_sigma_grad_t<double>(gotf, band, n, otf, xi, nax, grad_sigma, part, st);
}

}  // namespace dm
