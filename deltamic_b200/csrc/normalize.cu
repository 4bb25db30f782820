// normalize_tensor (render.py:5-6) on the device and its adjoint:
//   out = ((t - min t) / (max t - min t) + c) / (1 + c)
// with min / max propagating NaN and their gradient shared evenly by tied
// elements, as torch's full min() / max() reductions do.  Two launches each way,
// HBM-bound streams; the reductions are deterministic (fixed per-block ranges,
// the last block folds the partials in block order).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "dm_common.cuh"
#include "meshft_internal.h"

namespace dm {
namespace {

constexpr int kNrmThreads = 256;
constexpr int kNrmMaxBlocks = 148 * 8;

struct NrmSum {
  double s1, s2;     // sum g, sum g * (t - min)
  long long c0, c1;  // elements equal to min / max
};

template <typename T>
struct NrmWs {
  unsigned int ticket;
  int pad;
  NrmSum fin;
};

int nrm_blocks(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 4 * kNrmThreads - 1) /
                                                         (4 * kNrmThreads), kNrmMaxBlocks));
}

template <typename T>
__device__ __forceinline__ T nan_min(T a, T b) {  // NaN wins, as torch.min does
  return (b < a || b != b) && a == a ? b : a;
}
template <typename T>
__device__ __forceinline__ T nan_max(T a, T b) {
  return (b > a || b != b) && a == a ? b : a;
}

template <typename T>
__device__ __forceinline__ T inf_v() { return (T)INFINITY; }

// Per-block min / max; the last block to finish folds the partials in block
// order and writes stats[0..1] = (min, max).
template <typename T>
__global__ void __launch_bounds__(kNrmThreads)
    k_nrm_minmax(const T* __restrict__ t, int64_t n, T* __restrict__ part,
                 NrmWs<T>* ws, T* __restrict__ stats) {
  __shared__ T smn[kNrmThreads / 32], smx[kNrmThreads / 32];
  __shared__ bool last;
  T mn = inf_v<T>(), mx = -inf_v<T>();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T v = __ldg(t + i);
    mn = nan_min(mn, v);
    mx = nan_max(mx, v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = nan_min(mn, __shfl_down_sync(0xffffffffu, mn, o));
    mx = nan_max(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    smn[w] = mn;
    smx[w] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kNrmThreads / 32; ++k) {
      mn = nan_min(mn, smn[k]);
      mx = nan_max(mx, smx[k]);
    }
    part[2 * blockIdx.x] = mn;
    part[2 * blockIdx.x + 1] = mx;
    __threadfence();
    last = atomicAdd(&ws->ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  mn = inf_v<T>();
  mx = -inf_v<T>();
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
    mn = nan_min(mn, __ldcg(part + 2 * b));
    mx = nan_max(mx, __ldcg(part + 2 * b + 1));
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = nan_min(mn, __shfl_down_sync(0xffffffffu, mn, o));
    mx = nan_max(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    smn[w] = mn;
    smx[w] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kNrmThreads / 32; ++k) {
      mn = nan_min(mn, smn[k]);
      mx = nan_max(mx, smx[k]);
    }
    stats[0] = mn;
    stats[1] = mx;
    ws->ticket = 0;
  }
}

// The operation order of the eager expression on a CUDA tensor: (t - lo),
// / (hi - lo), + c, then the division by the scalar 1 + c done as a product with
// its reciprocal (as torch does for a host scalar divisor), each rounded in T.
template <typename T>
__global__ void __launch_bounds__(kNrmThreads)
    k_nrm_apply(const T* __restrict__ t, int64_t n, const T* __restrict__ stats, T c, T inv_d,
                T* __restrict__ out) {
  const T lo = stats[0], r = stats[1] - stats[0];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = ((__ldg(t + i) - lo) / r + c) * inv_d;
}

// Sums for the min / max terms of the adjoint and the tie counts.
template <typename T>
__global__ void __launch_bounds__(kNrmThreads)
    k_nrm_bsum(const T* __restrict__ t, const T* __restrict__ g, int64_t n,
               const T* __restrict__ stats, NrmSum* __restrict__ part, NrmWs<T>* ws) {
  __shared__ NrmSum sh[kNrmThreads / 32];
  __shared__ bool last;
  const T lo = stats[0], hi = stats[1];
  const bool lo_nan = lo != lo, hi_nan = hi != hi;
  NrmSum r{0.0, 0.0, 0, 0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T v = __ldg(t + i), gi = __ldg(g + i);
    r.s1 += (double)gi;
    r.s2 += (double)gi * (double)(v - lo);
    r.c0 += (lo_nan ? v != v : v == lo) ? 1 : 0;
    r.c1 += (hi_nan ? v != v : v == hi) ? 1 : 0;
  }
  for (int o = 16; o > 0; o >>= 1) {
    r.s1 += __shfl_down_sync(0xffffffffu, r.s1, o);
    r.s2 += __shfl_down_sync(0xffffffffu, r.s2, o);
    r.c0 += __shfl_down_sync(0xffffffffu, r.c0, o);
    r.c1 += __shfl_down_sync(0xffffffffu, r.c1, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) sh[w] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kNrmThreads / 32; ++k) {
      r.s1 += sh[k].s1;
      r.s2 += sh[k].s2;
      r.c0 += sh[k].c0;
      r.c1 += sh[k].c1;
    }
    part[blockIdx.x] = r;
    __threadfence();
    last = atomicAdd(&ws->ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  NrmSum q{0.0, 0.0, 0, 0};
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
    q.s1 += __ldcg(&part[b].s1);
    q.s2 += __ldcg(&part[b].s2);
    q.c0 += __ldcg(&part[b].c0);
    q.c1 += __ldcg(&part[b].c1);
  }
  for (int o = 16; o > 0; o >>= 1) {
    q.s1 += __shfl_down_sync(0xffffffffu, q.s1, o);
    q.s2 += __shfl_down_sync(0xffffffffu, q.s2, o);
    q.c0 += __shfl_down_sync(0xffffffffu, q.c0, o);
    q.c1 += __shfl_down_sync(0xffffffffu, q.c1, o);
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[w] = q;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kNrmThreads / 32; ++k) {
      q.s1 += sh[k].s1;
      q.s2 += sh[k].s2;
      q.c0 += sh[k].c0;
      q.c1 += sh[k].c1;
    }
    ws->fin = q;
    ws->ticket = 0;
  }
}

// grad_t = (g * (1 / (1 + c))) / r plus, on elements tied at the min (max), an even
// share of dL/dmin (dL/dmax):
//   dL/dr = -S2 / ((1 + c) r^2), dL/dmin = -S1 / ((1 + c) r) - dL/dr, dL/dmax = dL/dr.
template <typename T>
__global__ void __launch_bounds__(kNrmThreads)
    k_nrm_bapply(const T* __restrict__ t, const T* __restrict__ g, int64_t n,
                 const T* __restrict__ stats, T inv_d, const NrmWs<T>* __restrict__ ws,
                 T* __restrict__ grad_t) {
  const T lo = stats[0], hi = stats[1];
  const T r = hi - lo;
  const bool lo_nan = lo != lo, hi_nan = hi != hi;
  const NrmSum f = ws->fin;
  const double dd = 1.0 / (double)inv_d, rr = (double)r;
  const double dr = -f.s2 / (dd * rr * rr);
  const double dmn = -f.s1 / (dd * rr) - dr, dmx = dr;
  const T a0 = f.c0 > 0 ? (T)(dmn / (double)f.c0) : (T)0;
  const T a1 = f.c1 > 0 ? (T)(dmx / (double)f.c1) : (T)0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T v = __ldg(t + i);
    T o = (__ldg(g + i) * inv_d) / r;
    if (lo_nan ? v != v : v == lo) o += a0;
    if (hi_nan ? v != v : v == hi) o += a1;
    grad_t[i] = o;
  }
}

template <typename T>
size_t nrm_ws_bytes(int64_t n) {
  const size_t nb = (size_t)nrm_blocks(n);
  return 256 + nb * std::max(2 * sizeof(T), sizeof(NrmSum));
}

template <typename T>
int nrm_forward(const T* t, int64_t n, double contrast, T* out, T* stats, void* wsv,
                size_t ws_bytes, cudaStream_t st) {
  if (!t || !stats || !wsv || n <= 0) return DM_ERR_INVALID_ARG;
  if (ws_bytes < nrm_ws_bytes<T>(n)) return DM_ERR_WORKSPACE;
  NrmWs<T>* ws = (NrmWs<T>*)wsv;
  T* part = (T*)((char*)wsv + 256);
  const int nb = nrm_blocks(n);
  if (cudaMemsetAsync(ws, 0, sizeof(NrmWs<T>), st) != cudaSuccess) return DM_ERR_CUDA;
  k_nrm_minmax<T><<<nb, kNrmThreads, 0, st>>>(t, n, part, ws, stats);
  int launches = 1;
  if (out) {
    k_nrm_apply<T><<<nb, kNrmThreads, 0, st>>>(t, n, stats, (T)contrast,
                                               (T)1 / (T)(1.0 + contrast), out);
    ++launches;
  }
  count_launches(launches);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

template <typename T>
int nrm_backward(const T* t, const T* grad_out, int64_t n, double contrast, const T* stats,
                 T* grad_t, void* wsv, size_t ws_bytes, cudaStream_t st) {
  if (!t || !grad_out || !stats || !grad_t || !wsv || n <= 0) return DM_ERR_INVALID_ARG;
  if (ws_bytes < nrm_ws_bytes<T>(n)) return DM_ERR_WORKSPACE;
  NrmWs<T>* ws = (NrmWs<T>*)wsv;
  NrmSum* part = (NrmSum*)((char*)wsv + 256);
  const int nb = nrm_blocks(n);
  if (cudaMemsetAsync(ws, 0, sizeof(NrmWs<T>), st) != cudaSuccess) return DM_ERR_CUDA;
  k_nrm_bsum<T><<<nb, kNrmThreads, 0, st>>>(t, grad_out, n, stats, part, ws);
  k_nrm_bapply<T><<<nb, kNrmThreads, 0, st>>>(t, grad_out, n, stats,
                                              (T)1 / (T)(1.0 + contrast), ws, grad_t);
  count_launches(2);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

}  // namespace
}  // namespace dm

extern "C" {

size_t dm_normalize_workspace_size(int64_t n) {
  return n > 0 ? dm::nrm_ws_bytes<double>(n) : 0;
}

int dm_normalize(const float* t, int64_t n, double contrast, float* out, float* stats,
                 void* workspace, size_t ws_bytes, dm_stream_t stream) {
  return dm::nrm_forward<float>(t, n, contrast, out, stats, workspace, ws_bytes,
                                (cudaStream_t)stream);
}

int dm_normalize_backward(const float* t, const float* grad_out, int64_t n, double contrast,
                          const float* stats, float* grad_t, void* workspace, size_t ws_bytes,
                          dm_stream_t stream) {
  return dm::nrm_backward<float>(t, grad_out, n, contrast, stats, grad_t, workspace, ws_bytes,
                                 (cudaStream_t)stream);
}

int dm_normalize64(const double* t, int64_t n, double contrast, double* out, double* stats,
                   void* workspace, size_t ws_bytes, dm_stream_t stream) {
  return dm::nrm_forward<double>(t, n, contrast, out, stats, workspace, ws_bytes,
                                 (cudaStream_t)stream);
}

int dm_normalize64_backward(const double* t, const double* grad_out, int64_t n, double contrast,
                            const double* stats, double* grad_t, void* workspace,
                            size_t ws_bytes, dm_stream_t stream) {
  return dm::nrm_backward<double>(t, grad_out, n, contrast, stats, grad_t, workspace, ws_bytes,
                                  (cudaStream_t)stream);
}

}  // extern "C"
