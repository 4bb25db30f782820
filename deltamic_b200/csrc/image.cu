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

// Per-image state of dm_image_loss (one per segment of a batched call).
struct ImgWs {
  int err;
  int tie_count[2];   // recorded min / max ties (may exceed kTieSlots)
  int pad;
  ImgStats stats;
  double final_[3];   // loss, d_mn, d_mx
  int64_t cnt[2];
  int32_t ties[2][kTieSlots];
};
constexpr size_t kImgWsStride = ((sizeof(ImgWs) + 255) / 256) * 256;

// Segments of a launch: the images of the cells of a batch (CellDesc::grid_off
// and box shape), or one image [0, n0).  Each segment gets ``bps`` blocks.
struct Segs {
  const CellDesc* cells;
  int32_t nseg;
  int32_t bps;
  int64_t n0;
};

__device__ __forceinline__ void seg_range(const Segs& s, int seg, int64_t& b, int64_t& e) {
  if (s.cells) {
    const CellDesc& d = s.cells[seg];
    b = d.grid_off;
    e = b + (int64_t)d.n[0] * d.n[1] * d.n[2];
  } else {
    b = 0;
    e = s.n0;
  }
}

__device__ __forceinline__ float cabs(float2 z) { return sqrtf(fmaf(z.x, z.x, z.y * z.y)); }

int image_blocks(int64_t n) {
  const int64_t b = (n + kImgThreads - 1) / kImgThreads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 16));
}

static int blocks_per_segment(int64_t max_len, int nseg) {
  const int64_t b = (max_len + kImgThreads - 1) / kImgThreads;
  const int64_t cap = std::max<int64_t>(1, (int64_t)148 * 16 / std::max(nseg, 1));
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, cap));
}

size_t image_ws_bytes_segs(int64_t max_len, int nseg) {
  const size_t nb = (size_t)blocks_per_segment(max_len, nseg) * (size_t)std::max(nseg, 1);
  return 256 + kImgWsStride * (size_t)std::max(nseg, 1) + nb * sizeof(MinMaxPart) +
         nb * sizeof(LossPart);
}

size_t image_ws_bytes(int64_t n) { return image_ws_bytes_segs(n, 1); }

__device__ __forceinline__ void mm_merge(MinMaxPart& r, const MinMaxPart& o) {
  if (o.mn < r.mn || (o.mn == r.mn && o.imn < r.imn)) { r.mn = o.mn; r.imn = o.imn; }
  if (o.mx > r.mx || (o.mx == r.mx && o.imx < r.imx)) { r.mx = o.mx; r.imx = o.imx; }
}

__global__ void k_img_minmax(const float2* __restrict__ z, Segs sg, MinMaxPart* __restrict__ part) {
  __shared__ MinMaxPart sh[kImgThreads / 32];
  const int seg = blockIdx.x / sg.bps, loc = blockIdx.x % sg.bps;
  int64_t b, e;
  seg_range(sg, seg, b, e);
  MinMaxPart r{INFINITY, -INFINITY, INT64_MAX, INT64_MAX};
  for (int64_t i = b + (int64_t)loc * blockDim.x + threadIdx.x; i < e;
       i += (int64_t)sg.bps * blockDim.x) {
    const float a = cabs(z[i]);
    if (a < r.mn) { r.mn = a; r.imn = i; }
    if (a > r.mx) { r.mx = a; r.imx = i; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    MinMaxPart q;
    q.mn = __shfl_down_sync(0xffffffffu, r.mn, o);
    q.mx = __shfl_down_sync(0xffffffffu, r.mx, o);
    q.imn = __shfl_down_sync(0xffffffffu, r.imn, o);
    q.imx = __shfl_down_sync(0xffffffffu, r.imx, o);
    mm_merge(r, q);
  }
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    MinMaxPart t = sh[0];
    for (int w = 1; w < kImgThreads / 32; ++w) mm_merge(t, sh[w]);
    part[blockIdx.x] = t;
  }
}

// One block per segment: fixed strided subsets, then a fixed tree.
__global__ void k_img_minmax_final(const MinMaxPart* __restrict__ part, Segs sg, char* wsb) {
  __shared__ MinMaxPart sh[kImgThreads];
  const int seg = blockIdx.x;
  ImgWs* ws = (ImgWs*)(wsb + kImgWsStride * seg);
  MinMaxPart r{INFINITY, -INFINITY, INT64_MAX, INT64_MAX};
  for (int b = threadIdx.x; b < sg.bps; b += blockDim.x) mm_merge(r, part[seg * sg.bps + b]);
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
__global__ void k_img_loss(const float2* __restrict__ z, Segs sg, int kind,
                           const float* __restrict__ target, float contrast,
                           float* __restrict__ image, float2* __restrict__ grad_z, char* wsb,
                           LossPart* __restrict__ part) {
  __shared__ double sh[3][kImgThreads / 32];
  __shared__ long long shc[2][kImgThreads / 32];
  const int seg = blockIdx.x / sg.bps, loc = blockIdx.x % sg.bps;
  int64_t b, e;
  seg_range(sg, seg, b, e);
  ImgWs* ws = (ImgWs*)(wsb + kImgWsStride * seg);
  const float mn = ws->stats.mn, mx = ws->stats.mx;
  const float rng = mx - mn;
  const float inv = 1.0f / (rng * (1.0f + contrast));
  const float nseg_inv = 1.0f / (float)(e - b);
  double L = 0.0, dmn = 0.0, dmx = 0.0;
  long long cmn = 0, cmx = 0;
  for (int64_t i = b + (int64_t)loc * blockDim.x + threadIdx.x; i < e;
       i += (int64_t)sg.bps * blockDim.x) {
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
      gn = 2.0f * dlt * nseg_inv;
    }
    dmn += (double)gn * (-(1.0 - (double)u));
    dmx += (double)gn * (-(double)u);
    if (image) image[i] = a;
    if (grad_z) {
      const float g = gn * inv;
      const float sc = a > 0.f ? g / a : 0.f;
      grad_z[i] = make_float2(sc * zi.x, sc * zi.y);
    }
    if (a == mn) {
      ++cmn;
      const int slot = atomicAdd(&ws->tie_count[0], 1);
      if (slot < kTieSlots) ws->ties[0][slot] = (int32_t)(i - b);
    }
    if (a == mx) {
      ++cmx;
      const int slot = atomicAdd(&ws->tie_count[1], 1);
      if (slot < kTieSlots) ws->ties[1][slot] = (int32_t)(i - b);
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

// One block per segment: loss value, then the min/max gradient shared evenly by
// tied elements.
__global__ void k_img_final(const float2* __restrict__ z, Segs sg, int kind, float contrast,
                            const LossPart* __restrict__ part, char* wsb,
                            float* __restrict__ loss, float2* __restrict__ grad_z) {
  __shared__ double fin[3];
  __shared__ long long cnt[2];
  __shared__ LossPart sh[256];
  const int seg = blockIdx.x;
  int64_t b, e;
  seg_range(sg, seg, b, e);
  ImgWs* ws = (ImgWs*)(wsb + kImgWsStride * seg);
  {
    LossPart r{0, 0, 0, 0, 0};
    for (int k = threadIdx.x; k < sg.bps; k += blockDim.x) {
      const LossPart& q = part[seg * sg.bps + k];
      r.loss += q.loss;
      r.dmn += q.dmn;
      r.dmx += q.dmx;
      r.cmn += q.cmn;
      r.cmx += q.cmx;
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
    fin[0] = kind == 0 ? r.loss : r.loss / (double)(e - b);
    fin[1] = r.dmn * inv;
    fin[2] = r.dmx * inv;
    cnt[0] = r.cmn;
    cnt[1] = r.cmx;
    loss[seg] = (float)fin[0];
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
      const int64_t i = b + ws->ties[k][t];
      const float2 zi = z[i];
      const float a = cabs(zi);
      const float sc = a > 0.f ? add / a : 0.f;
      grad_z[i].x += sc * zi.x;
      grad_z[i].y += sc * zi.y;
    }
    __syncthreads();
  }
}

// Only when more than kTieSlots elements tie at a segment's min or max:
// distribute over that whole image (blocks of other segments return at once).
__global__ void k_img_ties_full(const float2* __restrict__ z, Segs sg, const char* wsb,
                                float2* __restrict__ grad_z) {
  const int seg = blockIdx.x / sg.bps, loc = blockIdx.x % sg.bps;
  const ImgWs* ws = (const ImgWs*)(wsb + kImgWsStride * seg);
  const bool over0 = ws->cnt[0] > kTieSlots, over1 = ws->cnt[1] > kTieSlots;
  if (!over0 && !over1) return;
  int64_t b, e;
  seg_range(sg, seg, b, e);
  const float mn = ws->stats.mn, mx = ws->stats.mx;
  const float add0 = over0 ? (float)(ws->final_[1] / (double)ws->cnt[0]) : 0.f;
  const float add1 = over1 ? (float)(ws->final_[2] / (double)ws->cnt[1]) : 0.f;
  for (int64_t i = b + (int64_t)loc * blockDim.x + threadIdx.x; i < e;
       i += (int64_t)sg.bps * blockDim.x) {
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

static int launch_image_loss_segs(const float2* z, const Segs& sg, int kind, const float* target,
                                  float contrast, float* image, float* loss, float2* grad_z,
                                  void* wsv, cudaStream_t st) {
  const int nb = sg.nseg * sg.bps;
  char* wsb = (char*)wsv + 256;
  MinMaxPart* mm = (MinMaxPart*)(wsb + kImgWsStride * sg.nseg);
  LossPart* lp = (LossPart*)(mm + nb);
  k_img_minmax<<<nb, kImgThreads, 0, st>>>(z, sg, mm);
  k_img_minmax_final<<<sg.nseg, kImgThreads, 0, st>>>(mm, sg, wsb);
  k_img_loss<<<nb, kImgThreads, 0, st>>>(z, sg, kind, target, contrast, image, grad_z, wsb, lp);
  k_img_final<<<sg.nseg, 256, 0, st>>>(z, sg, kind, contrast, lp, wsb, loss, grad_z);
  if (grad_z) k_img_ties_full<<<nb, kImgThreads, 0, st>>>(z, sg, wsb, grad_z);
  count_launches(4 + (grad_z ? 1 : 0));
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

int launch_image_loss(const float2* z, int64_t n, int kind, const float* target, float contrast,
                      float* image, float* loss, float2* grad_z, void* wsv, cudaStream_t st) {
  Segs sg{nullptr, 1, blocks_per_segment(n, 1), n};
  return launch_image_loss_segs(z, sg, kind, target, contrast, image, loss, grad_z, wsv, st);
}

int launch_image_loss_cells(const CellDesc* cells, int ncells, int64_t max_len, const float2* z,
                            int kind, const float* target, float contrast, float* image,
                            float* loss, float2* grad_z, void* wsv, cudaStream_t st) {
  Segs sg{cells, ncells, blocks_per_segment(max_len, ncells), 0};
  return launch_image_loss_segs(z, sg, kind, target, contrast, image, loss, grad_z, wsv, st);
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
