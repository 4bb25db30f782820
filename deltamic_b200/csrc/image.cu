// Fused image stage after the inverse FFT: |z| (render_image_from_ftmesh,
// render.py:177-180), normalize_tensor (render.py:5-6), loss and dL/dz; plus a
// plain Adam step for the fitting loop.  All HBM-bound streams.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "band_internal.h"
#include "dm_common.cuh"

namespace dm {

constexpr int kImgThreads = 256;

struct MinMaxPart {
  float mn, mx;
  int64_t imn, imx;
};

struct LossPart {
  double loss, dmn, dmx;
  int64_t cmn, cmx;
};

// Workspace of dm_image_loss.
struct ImgWs {
  int err;
  int tie_count[2];   // recorded min / max ties (may exceed kTieSlots)
  int pad;
  ImgStats stats;
  double final_[3];   // loss, d_mn, d_mx
  int64_t cnt[2];
  int32_t ties[2][kTieSlots];
};

__device__ __forceinline__ float cabs(float2 z) { return sqrtf(fmaf(z.x, z.x, z.y * z.y)); }

int image_blocks(int64_t n) {
  const int64_t b = (n + kImgThreads - 1) / kImgThreads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 16));
}

size_t image_ws_bytes(int64_t n) {
  const size_t nb = (size_t)image_blocks(n);
  return 256 + ((sizeof(ImgWs) + 255) / 256) * 256 + nb * sizeof(MinMaxPart) + nb * sizeof(LossPart);
}

__global__ void k_img_minmax(const float2* __restrict__ z, int64_t n, MinMaxPart* __restrict__ part) {
  __shared__ MinMaxPart sh[kImgThreads / 32];
  float mn = INFINITY, mx = -INFINITY;
  int64_t imn = INT64_MAX, imx = INT64_MAX;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float a = cabs(z[i]);
    if (a < mn) { mn = a; imn = i; }
    if (a > mx) { mx = a; imx = i; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const float omn = __shfl_down_sync(0xffffffffu, mn, o);
    const float omx = __shfl_down_sync(0xffffffffu, mx, o);
    const int64_t oimn = __shfl_down_sync(0xffffffffu, imn, o);
    const int64_t oimx = __shfl_down_sync(0xffffffffu, imx, o);
    if (omn < mn || (omn == mn && oimn < imn)) { mn = omn; imn = oimn; }
    if (omx > mx || (omx == mx && oimx < imx)) { mx = omx; imx = oimx; }
  }
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = MinMaxPart{mn, mx, imn, imx};
  __syncthreads();
  if (threadIdx.x == 0) {
    MinMaxPart r = sh[0];
    for (int w = 1; w < kImgThreads / 32; ++w) {
      const MinMaxPart o = sh[w];
      if (o.mn < r.mn || (o.mn == r.mn && o.imn < r.imn)) { r.mn = o.mn; r.imn = o.imn; }
      if (o.mx > r.mx || (o.mx == r.mx && o.imx < r.imx)) { r.mx = o.mx; r.imx = o.imx; }
    }
    part[blockIdx.x] = r;
  }
}

__device__ __forceinline__ void mm_merge(MinMaxPart& r, const MinMaxPart& o) {
  if (o.mn < r.mn || (o.mn == r.mn && o.imn < r.imn)) { r.mn = o.mn; r.imn = o.imn; }
  if (o.mx > r.mx || (o.mx == r.mx && o.imx < r.imx)) { r.mx = o.mx; r.imx = o.imx; }
}

// One block: each thread merges a fixed strided subset, then a fixed tree.
__global__ void k_img_minmax_final(const MinMaxPart* __restrict__ part, int nb, ImgWs* ws) {
  __shared__ MinMaxPart sh[kImgThreads];
  MinMaxPart r{INFINITY, -INFINITY, INT64_MAX, INT64_MAX};
  for (int b = threadIdx.x; b < nb; b += blockDim.x) mm_merge(r, part[b]);
  sh[threadIdx.x] = r;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) mm_merge(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    ws->stats = ImgStats{sh[0].mn, sh[0].mx, sh[0].imn, sh[0].imx};
    ws->tie_count[0] = 0;
    ws->tie_count[1] = 0;
  }
}

// Per element: normalised value, loss term, dL/dimage without the min/max
// terms, dL/dz = g z/|z|; partial sums of the loss and of the min/max terms.
__global__ void k_img_loss(const float2* __restrict__ z, int64_t n, int kind,
                           const float* __restrict__ target, float contrast,
                           float* __restrict__ image, float2* __restrict__ grad_z, ImgWs* ws,
                           LossPart* __restrict__ part) {
  __shared__ double sh[3][kImgThreads / 32];
  __shared__ long long shc[2][kImgThreads / 32];
  const float mn = ws->stats.mn, mx = ws->stats.mx;
  const float rng = mx - mn;
  const float inv = 1.0f / (rng * (1.0f + contrast));
  double L = 0.0, dmn = 0.0, dmx = 0.0;
  long long cmn = 0, cmx = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float2 zi = z[i];
    const float a = cabs(zi);
    const float u = (a - mn) / rng;
    const float nv = (u + contrast) / (1.0f + contrast);
    float gn;
    if (kind == 0) {
      L += nv;
      gn = 1.0f;
    } else {
      const float dlt = nv - target[i];
      L += (double)dlt * dlt;
      gn = 2.0f * dlt / (float)n;
    }
    dmn += (double)gn * (-(1.0 - (double)u));
    dmx += (double)gn * (-(double)u);
    if (image) image[i] = a;
    if (grad_z) {
      const float g = gn * inv;
      const float s = a > 0.f ? g / a : 0.f;
      grad_z[i] = make_float2(s * zi.x, s * zi.y);
    }
    if (a == mn) {
      ++cmn;
      const int slot = atomicAdd(&ws->tie_count[0], 1);
      if (slot < kTieSlots) ws->ties[0][slot] = (int32_t)i;
    }
    if (a == mx) {
      ++cmx;
      const int slot = atomicAdd(&ws->tie_count[1], 1);
      if (slot < kTieSlots) ws->ties[1][slot] = (int32_t)i;
    }
  }
  double v[3] = {L, dmn, dmx};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double x = v[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = x;
  }
  long long c[2] = {cmn, cmx};
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    long long x = c[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) shc[k][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    LossPart r{0, 0, 0, 0, 0};
    for (int w = 0; w < kImgThreads / 32; ++w) {
      r.loss += sh[0][w];
      r.dmn += sh[1][w];
      r.dmx += sh[2][w];
      r.cmn += shc[0][w];
      r.cmx += shc[1][w];
    }
    part[blockIdx.x] = r;
  }
}

// Loss value, then the min/max gradient shared evenly by tied elements.
__global__ void k_img_final(const float2* __restrict__ z, int64_t n, int kind, float contrast,
                            const LossPart* __restrict__ part, int nb, ImgWs* ws,
                            float* __restrict__ loss, float2* __restrict__ grad_z) {
  __shared__ double fin[3];
  __shared__ long long cnt[2];
  __shared__ LossPart sh[256];
  {
    LossPart r{0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      r.loss += part[b].loss;
      r.dmn += part[b].dmn;
      r.dmx += part[b].dmx;
      r.cmn += part[b].cmn;
      r.cmx += part[b].cmx;
    }
    sh[threadIdx.x] = r;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) {
        sh[threadIdx.x].loss += sh[threadIdx.x + o].loss;
        sh[threadIdx.x].dmn += sh[threadIdx.x + o].dmn;
        sh[threadIdx.x].dmx += sh[threadIdx.x + o].dmx;
        sh[threadIdx.x].cmn += sh[threadIdx.x + o].cmn;
        sh[threadIdx.x].cmx += sh[threadIdx.x + o].cmx;
      }
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) {
    const LossPart r = sh[0];
    const double rng = (double)ws->stats.mx - (double)ws->stats.mn;
    const double inv = 1.0 / (rng * (1.0 + contrast));
    fin[0] = kind == 0 ? r.loss : r.loss / (double)n;
    fin[1] = r.dmn * inv;
    fin[2] = r.dmx * inv;
    cnt[0] = r.cmn;
    cnt[1] = r.cmx;
    *loss = (float)fin[0];
    ws->final_[0] = fin[0];
    ws->final_[1] = fin[1];
    ws->final_[2] = fin[2];
    ws->cnt[0] = r.cmn;
    ws->cnt[1] = r.cmx;
  }
  __syncthreads();
  if (!grad_z) return;
  for (int k = 0; k < 2; ++k) {
    const long long c = cnt[k];
    if (c <= 0 || c > kTieSlots) continue;  // overflow handled by k_img_ties_full
    const float add = (float)(fin[1 + k] / (double)c);
    for (int t = threadIdx.x; t < c; t += blockDim.x) {
      const int32_t i = ws->ties[k][t];
      const float2 zi = z[i];
      const float a = cabs(zi);
      const float s = a > 0.f ? add / a : 0.f;
      grad_z[i].x += s * zi.x;
      grad_z[i].y += s * zi.y;
    }
    __syncthreads();
  }
}

// Only when more than kTieSlots elements tie at the min or max: distribute over
// the whole image (the kernel returns at once otherwise).
__global__ void k_img_ties_full(const float2* __restrict__ z, int64_t n, const ImgWs* ws,
                                float2* __restrict__ grad_z) {
  const bool over0 = ws->cnt[0] > kTieSlots, over1 = ws->cnt[1] > kTieSlots;
  if (!over0 && !over1) return;
  const float mn = ws->stats.mn, mx = ws->stats.mx;
  const float add0 = over0 ? (float)(ws->final_[1] / (double)ws->cnt[0]) : 0.f;
  const float add1 = over1 ? (float)(ws->final_[2] / (double)ws->cnt[1]) : 0.f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float2 zi = z[i];
    const float a = cabs(zi);
    float add = 0.f;
    if (over0 && a == mn) add += add0;
    if (over1 && a == mx) add += add1;
    if (add != 0.f && a > 0.f) {
      grad_z[i].x += add / a * zi.x;
      grad_z[i].y += add / a * zi.y;
    }
  }
}

int launch_image_loss(const float2* z, int64_t n, int kind, const float* target, float contrast,
                      float* image, float* loss, float2* grad_z, void* wsv, cudaStream_t st) {
  const int nb = image_blocks(n);
  char* base = (char*)wsv + 256;
  ImgWs* ws = (ImgWs*)base;
  MinMaxPart* mm = (MinMaxPart*)(base + ((sizeof(ImgWs) + 255) / 256) * 256);
  LossPart* lp = (LossPart*)(mm + nb);
  k_img_minmax<<<nb, kImgThreads, 0, st>>>(z, n, mm);
  k_img_minmax_final<<<1, kImgThreads, 0, st>>>(mm, nb, ws);
  k_img_loss<<<nb, kImgThreads, 0, st>>>(z, n, kind, target, contrast, image, grad_z, ws, lp);
  k_img_final<<<1, 256, 0, st>>>(z, n, kind, contrast, lp, nb, ws, loss, grad_z);
  if (grad_z) k_img_ties_full<<<nb, kImgThreads, 0, st>>>(z, n, ws, grad_z);
  count_launches(4 + (grad_z ? 1 : 0));
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// Adam (torch.optim.Adam, no weight decay / amsgrad).  One block for small
// arrays so the step counter can be bumped after every thread has read it.

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps,
                       int64_t* step, int bump) {
  const int64_t t = *step + 1;
  const double bc1 = 1.0 - pow((double)b1, (double)t);
  const double bc2s = sqrt(1.0 - pow((double)b2, (double)t));
  const float step_size = (float)(lr / bc1);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float den = sqrtf(vi) / (float)bc2s + eps;
    p[i] -= step_size * mi / den;
  }
  if (bump) {
    __syncthreads();
    if (threadIdx.x == 0) *step = t;
  }
}

__global__ void k_bump(int64_t* step) { *step += 1; }

int launch_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1,
                float b2, float eps, int64_t* step, cudaStream_t st) {
  if (n <= 4096) {
    k_adam<<<1, 1024, 0, st>>>(p, g, m, v, n, lr, b1, b2, eps, step, 1);
    count_launches(1);
  } else {
    const int64_t nb = std::min<int64_t>((n + 255) / 256, 148 * 16);
    k_adam<<<(unsigned)nb, 256, 0, st>>>(p, g, m, v, n, lr, b1, b2, eps, step, 0);
    k_bump<<<1, 1, 0, st>>>(step);
    count_launches(2);
  }
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

}  // namespace dm
