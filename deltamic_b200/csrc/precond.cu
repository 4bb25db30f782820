// Gradient preconditioning and the vector Adam step of the preconditioned fit.
//
// The reference's fitting notebook replaces the vertex gradient g by
// (M^2)^-1 g with M = I + lambda L (L the uniform mesh Laplacian; largesteps'
// compute_matrix + CholeskySolver(M@M), Examples/Gradient_Descent.ipynb cell 2),
// and its optimize.py:207-212 forms the same operator densely as
// inv(M) @ inv(M).  Here the dense operator P (nv x nv, float32, rows padded to a
// multiple of 4) is built once per topology and applied every step by an
// HBM-bound product: each warp streams eight rows of P with 16-byte loads (sixteen
// in flight per lane) and multiplies them with the matching 4 x 3 block of g, read
// through L1 as three 16-byte loads.
// For meshes whose dense operator would not fit (or stream) well, the sparse form
// below applies the same operator without forming it.
// The optimizer is VectorAdam of optimize.py:215-258 (axis -1): the second
// moment of each vertex is the squared norm of its 3-vector gradient.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "band_internal.h"
#include "dm_common.cuh"

namespace dm {
namespace {

constexpr int kRowsPerWarp = 8;
constexpr int kGemvThreads = 128;

// out[r][d] = sum_c P[r][c] g[c][d] for d < 3; P row stride ldp (multiple of 4),
// g and out [nv][3] (g read through the read-only cache).
__global__ void __launch_bounds__(kGemvThreads)
    k_precond_gemv(const float* __restrict__ P, int64_t nv, int64_t ldp,
                   const float* __restrict__ g, float* __restrict__ out, bool g16) {
  const int64_t warp = ((int64_t)blockIdx.x * kGemvThreads + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t r0 = warp * kRowsPerWarp;
  if (r0 >= nv) return;
  float acc[kRowsPerWarp][3];
#pragma unroll
  for (int i = 0; i < kRowsPerWarp; ++i) acc[i][0] = acc[i][1] = acc[i][2] = 0.f;
  const int64_t nq = ldp / 4;  // 16-byte column groups per row
  const int nrow = (int)min((int64_t)kRowsPerWarp, nv - r0);
  // two column groups per lane and round: eight 16-byte row loads in flight
  for (int64_t q0 = lane; q0 < nq; q0 += 64) {
    float4 pr[2][kRowsPerWarp];
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int i = 0; i < kRowsPerWarp; ++i) {
        const int64_t q = q0 + 32 * u;
        pr[u][i] = (q < nq && i < nrow)
                       ? __ldcs(reinterpret_cast<const float4*>(P + (r0 + i) * ldp) + q)
                       : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int64_t c = 4 * (q0 + 32 * u);
      float gv[12];
      if (c + 4 <= nv && g16) {
        // g[c..c+3][0..2]: twelve floats at a 48c-byte offset, three 16-byte loads
        const float4* g4 = reinterpret_cast<const float4*>(g + 3 * c);
        const float4 a = __ldg(g4), b = __ldg(g4 + 1), e = __ldg(g4 + 2);
        gv[0] = a.x; gv[1] = a.y; gv[2] = a.z; gv[3] = a.w;
        gv[4] = b.x; gv[5] = b.y; gv[6] = b.z; gv[7] = b.w;
        gv[8] = e.x; gv[9] = e.y; gv[10] = e.z; gv[11] = e.w;
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const bool live = c + k < nv;
          gv[3 * k + 0] = live ? __ldg(g + 3 * (c + k) + 0) : 0.f;
          gv[3 * k + 1] = live ? __ldg(g + 3 * (c + k) + 1) : 0.f;
          gv[3 * k + 2] = live ? __ldg(g + 3 * (c + k) + 2) : 0.f;
        }
      }
#pragma unroll
      for (int i = 0; i < kRowsPerWarp; ++i) {
        const float pv[4] = {pr[u][i].x, pr[u][i].y, pr[u][i].z, pr[u][i].w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          acc[i][0] = fmaf(pv[k], gv[3 * k + 0], acc[i][0]);
          acc[i][1] = fmaf(pv[k], gv[3 * k + 1], acc[i][1]);
          acc[i][2] = fmaf(pv[k], gv[3 * k + 2], acc[i][2]);
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < kRowsPerWarp; ++i)
#pragma unroll
    for (int d = 0; d < 3; ++d)
      for (int o = 16; o > 0; o >>= 1) acc[i][d] += __shfl_xor_sync(0xffffffffu, acc[i][d], o);
  if (lane < kRowsPerWarp * 3) {  // 24 lanes write the 8 x 3 outputs
    const int i = lane / 3, d = lane % 3;
    if (r0 + i < nv) {
      float v = 0.f;
#pragma unroll
      for (int ii = 0; ii < kRowsPerWarp; ++ii)
#pragma unroll
        for (int dd = 0; dd < 3; ++dd)
          if (ii == i && dd == d) v = acc[ii][dd];
      out[3 * (r0 + i) + d] = v;
    }
  }
}

// VectorAdam (optimize.py:215-258, axis -1) on nv 3-vectors; ``step`` is a device
// counter, incremented by the single-block launch or by k_step_bump afterwards.
__global__ void k_vector_adam(float* __restrict__ p, const float* __restrict__ g,
                              float* __restrict__ m, float* __restrict__ v, int64_t nv, float lr,
                              float b1, float b2, float eps, int64_t* step, int bump) {
  const int64_t t = *step + 1;
  const double bc1 = 1.0 - pow((double)b1, (double)t);
  const double bc2 = 1.0 - pow((double)b2, (double)t);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float g0 = g[3 * i], g1 = g[3 * i + 1], g2 = g[3 * i + 2];
    const float nrm = sqrtf(g0 * g0 + g1 * g1 + g2 * g2);
    const float vi = b2 * v[i] + (1.0f - b2) * (nrm * nrm);
    v[i] = vi;
    const float den = eps + sqrtf((float)(vi / bc2));
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float mi = b1 * m[3 * i + d] + (1.0f - b1) * g[3 * i + d];
      m[3 * i + d] = mi;
      p[3 * i + d] -= lr * ((float)(mi / bc1) / den);
    }
  }
  if (bump) {
    __syncthreads();
    if (threadIdx.x == 0) *step = t;
  }
}

__global__ void k_step_bump(int64_t* step) { *step += 1; }

// Sparse form: (M M)^-1 g as two solves with M = I + lambda L, each a Chebyshev
// iteration for the eigenvalue interval [theta - delta, theta + delta] of M (Saad,
// Iterative Methods for Sparse Linear Systems, Alg. 12.1):
//   x0 = 0, r0 = b, d0 = r0 / theta, rho0 = delta / theta;
//   x_{k+1} = x_k + d_k,  r_{k+1} = r_k - M d_k,
//   d_{k+1} = rho_{k+1} rho_k d_k + (2 rho_{k+1} / delta) r_{k+1},
//   rho_{k+1} = 1 / (2 theta / delta - rho_k).
// L is held as CSR neighbour lists (row i: the vertices sharing an edge with i), so
// (M d)_i = (1 + lambda deg_i) d_i - lambda sum_j d_j.  One launch per iteration
// (no device-side waits); the rho sequence is fixed by the interval, so the
// launches carry their coefficients and replay in a CUDA graph.

__global__ void k_cheb_init(const float* __restrict__ b, int64_t n3, float inv_theta,
                            float* __restrict__ x, float* __restrict__ r,
                            float* __restrict__ d) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float v = b[i];
    x[i] = 0.f;
    r[i] = v;
    d[i] = v * inv_theta;
  }
}

__global__ void k_cheb_iter(const int32_t* __restrict__ rowp, const int32_t* __restrict__ col,
                            int64_t nv, float lam, float a, float c,
                            const float* __restrict__ dc, float* __restrict__ dn,
                            float* __restrict__ r, float* __restrict__ x) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t b = rowp[i], e = rowp[i + 1];
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
    for (int32_t k = b; k < e; ++k) {
      const int64_t j = 3 * (int64_t)col[k];
      s0 += dc[j];
      s1 += dc[j + 1];
      s2 += dc[j + 2];
    }
    const float w = fmaf(lam, (float)(e - b), 1.0f);
    const float s[3] = {s0, s1, s2};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int64_t o = 3 * i + q;
      const float di = dc[o];
      const float md = fmaf(w, di, -lam * s[q]);
      x[o] += di;
      const float ri = r[o] - md;
      r[o] = ri;
      dn[o] = fmaf(a, di, c * ri);
    }
  }
}

}  // namespace
}  // namespace dm

using namespace dm;

extern "C" {

int dm_precond_apply(const float* P, int64_t nv, int64_t ldp, const float* grad, float* out,
                     dm_stream_t stream) {
  if (nv < 0 || ldp < nv || (ldp & 3) != 0) return DM_ERR_INVALID_ARG;
  if (nv == 0) return DM_OK;
  if (!P || !grad || !out || grad == out) return DM_ERR_INVALID_ARG;
  if (((uintptr_t)P & 15) != 0) return DM_ERR_INVALID_ARG;
  const int64_t warps = (nv + kRowsPerWarp - 1) / kRowsPerWarp;
  const int64_t blocks = (warps * 32 + kGemvThreads - 1) / kGemvThreads;
  if (blocks > INT32_MAX) return DM_ERR_SIZE;
  k_precond_gemv<<<(unsigned)blocks, kGemvThreads, 0, (cudaStream_t)stream>>>(
      P, nv, ldp, grad, out, ((uintptr_t)grad & 15) == 0);
  count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

int dm_precond_chebyshev(const int32_t* rowp, const int32_t* col, int64_t nv, float lambda,
                         double lo, double hi, int iters, const float* grad, float* out,
                         float* work, dm_stream_t stream) {
  if (nv < 0 || iters < 1 || iters > 4096 || !(lambda >= 0.f) || !(lo > 0.0) || !(hi >= lo))
    return DM_ERR_INVALID_ARG;
  if (nv == 0) return DM_OK;
  if (!rowp || !col || !grad || !out || !work || grad == out) return DM_ERR_INVALID_ARG;
  if (3 * nv > (int64_t)INT32_MAX * 64) return DM_ERR_SIZE;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n3 = 3 * nv;
  float* y = work;          // the first solve's result
  float* r = work + n3;
  float* d0 = work + 2 * n3;
  float* d1 = work + 3 * n3;
  const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo);
  const unsigned nb3 = (unsigned)std::min<int64_t>((n3 + 255) / 256, 148 * 8);
  const unsigned nbv = (unsigned)std::min<int64_t>((nv + 127) / 128, 148 * 8);
  int launches = 0;
  for (int solve = 0; solve < 2; ++solve) {
    const float* b = solve == 0 ? grad : y;
    float* x = solve == 0 ? y : out;
    k_cheb_init<<<nb3, 256, 0, st>>>(b, n3, (float)(1.0 / theta), x, r, d0);
    ++launches;
    double rho = delta > 0.0 ? delta / theta : 0.0;
    float* dc = d0;
    float* dn = d1;
    for (int k = 0; k < iters; ++k) {
      double a = 0.0, c = 0.0;
      if (delta > 0.0) {
        const double rho1 = 1.0 / (2.0 * theta / delta - rho);
        a = rho1 * rho;
        c = 2.0 * rho1 / delta;
        rho = rho1;
      }
      k_cheb_iter<<<nbv, 128, 0, st>>>(rowp, col, nv, lambda, (float)a, (float)c, dc, dn, r, x);
      ++launches;
      std::swap(dc, dn);
    }
  }
  count_launches(launches);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

int dm_vector_adam_step(float* param, const float* grad, float* exp_avg, float* exp_avg_norm_sq,
                        int64_t nv, float lr, float beta1, float beta2, float eps, int64_t* step,
                        dm_stream_t stream) {
  if (nv < 0 || !step || (nv > 0 && (!param || !grad || !exp_avg || !exp_avg_norm_sq)))
    return DM_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (nv <= 4096) {
    k_vector_adam<<<1, 1024, 0, st>>>(param, grad, exp_avg, exp_avg_norm_sq, nv, lr, beta1, beta2,
                                      eps, step, 1);
    count_launches(1);
  } else {
    const int64_t nb = std::min<int64_t>((nv + 255) / 256, 148 * 16);
    k_vector_adam<<<(unsigned)nb, 256, 0, st>>>(param, grad, exp_avg, exp_avg_norm_sq, nv, lr,
                                                beta1, beta2, eps, step, 0);
    k_step_bump<<<1, 1, 0, st>>>(step);
    count_launches(2);
  }
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

}  // extern "C"
