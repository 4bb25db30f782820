// 3x3x3 stride-2 padding-1 3D convolutions (channels-last, BF16 operands, FP32
// accumulation on the tensor cores) with a fused bias + GELU epilogue, and their
// adjoints.  They run the learned initialiser's encoder (no counterpart in the
// reference).  All three products are implicit GEMMs over one generic tiled
// kernel with gather loaders:
//   forward  C[m, n]  = sum_k  A[m, k] W[k, n]       (A = im2col of x, on the fly)
//   wgrad    dW[k, n] = sum_m  A[m, k] dP[m, n]      (split over m, fixed-order sum)
//   dgrad    dX[q, c] = sum_t  dP[q(t)] W[t, c]      (one GEMM per stride parity
//                                                   class of the input voxel)
// with m = (b, od, oh, ow), k = ((kd*3 + kh)*3 + kw)*Ci + ci (rows past 27*Ci are
// zero padding up to a multiple of 32), P = pre-activation, dP = dL/dP.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <mma.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/deltamic_b200.h"
#include "band_internal.h"

namespace dm {

using bf16 = __nv_bfloat16;
using namespace nvcuda;

constexpr int kBM = 64, kBK = 32, kConvThreads = 128;

struct ConvShape {
  int B, D, H, W, Ci;      // input
  int Do, Ho, Wo, Co;      // output
  int K, Kp;               // 27*Ci and its padding to kBK
  int64_t M;               // B*Do*Ho*Wo
};

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) +
         x * expf(-0.5f * x * x) * 0.39894228040143268f;
}

// im2col element A[m, k] of x (zero outside the volume and in the K padding).
__device__ __forceinline__ bf16 im2col(const bf16* __restrict__ x, const ConvShape& s, int64_t m,
                                       int k) {
  if (k >= s.K) return __float2bfloat16(0.f);
  const int ci = k % s.Ci;
  const int tap = k / s.Ci;
  const int kw = tap % 3, kh = (tap / 3) % 3, kd = tap / 9;
  int64_t t = m;
  const int ow = (int)(t % s.Wo); t /= s.Wo;
  const int oh = (int)(t % s.Ho); t /= s.Ho;
  const int od = (int)(t % s.Do);
  const int b = (int)(t / s.Do);
  const int d = 2 * od - 1 + kd, h = 2 * oh - 1 + kh, w = 2 * ow - 1 + kw;
  if (d < 0 || d >= s.D || h < 0 || h >= s.H || w < 0 || w >= s.W) return __float2bfloat16(0.f);
  return x[((((int64_t)b * s.D + d) * s.H + h) * s.W + w) * s.Ci + ci];
}

// Generic tile: C[rows x BN] over a reduction [r_begin, r_end) split by blockIdx.y.
template <int BN, class LA, class LB, class EP>
__global__ void __launch_bounds__(kConvThreads) k_conv_gemm(LA la, LB lb, EP ep, int64_t rows,
                                                            int64_t red_total, int64_t red_split) {
  __shared__ __align__(32) bf16 As[kBM][kBK + 8];
  __shared__ __align__(32) bf16 Bs[kBK][BN + 8];
  __shared__ __align__(32) float Cs[kBM][BN + 4];
  const int64_t row0 = (int64_t)blockIdx.x * kBM;
  const int64_t r_begin = (int64_t)blockIdx.y * red_split;
  const int64_t r_end = min(red_total, r_begin + red_split);
  const int warp = threadIdx.x >> 5;
  wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[BN / 16];
#pragma unroll
  for (int j = 0; j < BN / 16; ++j) wmma::fill_fragment(acc[j], 0.0f);
  const bf16 zero = __float2bfloat16(0.f);
  for (int64_t k0 = r_begin; k0 < r_end; k0 += kBK) {
    for (int e = threadIdx.x; e < kBM * kBK; e += kConvThreads) {
      const int r = e / kBK, c = e % kBK;
      const int64_t row = row0 + r, red = k0 + c;
      As[r][c] = (row < rows && red < r_end) ? la(row, red) : zero;
    }
    for (int e = threadIdx.x; e < kBK * BN; e += kConvThreads) {
      const int r = e / BN, c = e % BN;
      const int64_t red = k0 + r;
      Bs[r][c] = red < r_end ? lb(red, c) : zero;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 16) {
      wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, wmma::row_major> a;
      wmma::load_matrix_sync(a, &As[warp * 16][kk], kBK + 8);
#pragma unroll
      for (int j = 0; j < BN / 16; ++j) {
        wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, wmma::row_major> b;
        wmma::load_matrix_sync(b, &Bs[kk][j * 16], BN + 8);
        wmma::mma_sync(acc[j], a, b, acc[j]);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < BN / 16; ++j)
    wmma::store_matrix_sync(&Cs[warp * 16][j * 16], acc[j], BN + 4, wmma::mem_row_major);
  __syncthreads();
  for (int e = threadIdx.x; e < kBM * BN; e += kConvThreads) {
    const int r = e / BN, c = e % BN;
    const int64_t row = row0 + r;
    if (row < rows) ep(row, c, (int)blockIdx.y, Cs[r][c]);
  }
}

// ---------------------------------------------------------------------------
// forward

struct FwdA {
  const bf16* x;
  ConvShape s;
  __device__ bf16 operator()(int64_t m, int64_t k) const { return im2col(x, s, m, (int)k); }
};
struct WeightB {  // W[k, n], row-major [Kp, Co]
  const bf16* w;
  int Co;
  __device__ bf16 operator()(int64_t k, int n) const { return w[k * Co + n]; }
};
struct FwdEp {
  const float* bias;
  float* pre;
  bf16* act;
  int Co;
  __device__ void operator()(int64_t m, int n, int, float v) const {
    const float p = v + (bias ? bias[n] : 0.f);
    pre[m * Co + n] = p;
    act[m * Co + n] = __float2bfloat16(gelu(p));
  }
};

// ---------------------------------------------------------------------------
// backward pieces

__global__ void k_gelu_back(const float* __restrict__ pre, const float* __restrict__ dact,
                            bf16* __restrict__ dpre, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dpre[i] = __float2bfloat16(dact[i] * gelu_grad(pre[i]));
}

struct WgradA {  // A^T[k, m]
  const bf16* x;
  ConvShape s;
  __device__ bf16 operator()(int64_t k, int64_t m) const { return im2col(x, s, m, (int)k); }
};
struct DpreB {  // dP[m, n]
  const bf16* dp;
  int Co;
  __device__ bf16 operator()(int64_t m, int n) const { return dp[m * Co + n]; }
};
struct WgradEp {  // partial[split][k][n]
  float* part;
  int64_t stride;  // Kp * Co
  int Co;
  __device__ void operator()(int64_t k, int n, int split, float v) const {
    part[split * stride + k * Co + n] = v;
  }
};

__global__ void k_sum_splits(const float* __restrict__ part, int splits, int64_t n,
                             float* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int k = 0; k < splits; ++k) s += part[k * n + i];
    out[i] = s;
  }
}

// db[n] = sum_m dP[m, n]: one block per n, fixed-order tree.
__global__ void k_bias_grad(const bf16* __restrict__ dp, int64_t M, int Co, float* __restrict__ db) {
  __shared__ float sh[256];
  const int n = blockIdx.x;
  float s = 0.f;
  for (int64_t m = threadIdx.x; m < M; m += blockDim.x) s += __bfloat162float(dp[m * Co + n]);
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[n] = sh[0];
}

// dgrad for the input voxels of one stride-parity class (pd, ph, pw): per axis an
// even coordinate d takes tap 1 (od = d/2), an odd one taps 0 and 2
// (od = (d+1)/2, (d-1)/2).
struct Cls {
  int p[3];     // parity per axis
  int n[3];     // class extent per axis
  int nt[3];    // taps per axis (1 or 2)
  int T;        // taps in the class
};

__device__ __forceinline__ void cls_tap(const Cls& c, int t, int kk[3]) {
  const int tw = t % c.nt[2], th = (t / c.nt[2]) % c.nt[1], td = t / (c.nt[2] * c.nt[1]);
  const int tt[3] = {td, th, tw};
#pragma unroll
  for (int a = 0; a < 3; ++a) kk[a] = c.p[a] == 0 ? 1 : (tt[a] == 0 ? 0 : 2);
}

struct DgradA {  // A[q, (tap, co)] = dP at the output voxel reached through the tap
  const bf16* dp;
  ConvShape s;
  Cls c;
  __device__ bf16 operator()(int64_t q, int64_t r) const {
    const int co = (int)(r % s.Co);
    const int t = (int)(r / s.Co);
    if (t >= c.T) return __float2bfloat16(0.f);
    int kk[3];
    cls_tap(c, t, kk);
    int64_t u = q;
    const int iw = (int)(u % c.n[2]); u /= c.n[2];
    const int ih = (int)(u % c.n[1]); u /= c.n[1];
    const int id = (int)(u % c.n[0]);
    const int b = (int)(u / c.n[0]);
    const int d = 2 * id + c.p[0], h = 2 * ih + c.p[1], w = 2 * iw + c.p[2];
    const int od = (d + 1 - kk[0]) >> 1, oh = (h + 1 - kk[1]) >> 1, ow = (w + 1 - kk[2]) >> 1;
    if (od < 0 || od >= s.Do || oh < 0 || oh >= s.Ho || ow < 0 || ow >= s.Wo)
      return __float2bfloat16(0.f);
    return dp[((((int64_t)b * s.Do + od) * s.Ho + oh) * s.Wo + ow) * s.Co + co];
  }
};
struct DgradB {  // B[(tap, co), ci] = W[(k(tap), ci), co]
  const bf16* w;
  ConvShape s;
  Cls c;
  __device__ bf16 operator()(int64_t r, int ci) const {
    const int co = (int)(r % s.Co);
    const int t = (int)(r / s.Co);
    if (t >= c.T || ci >= s.Ci) return __float2bfloat16(0.f);
    int kk[3];
    cls_tap(c, t, kk);
    const int tap = (kk[0] * 3 + kk[1]) * 3 + kk[2];
    return w[((int64_t)tap * s.Ci + ci) * s.Co + co];
  }
};
struct DgradEp {
  float* dx;
  ConvShape s;
  Cls c;
  __device__ void operator()(int64_t q, int ci, int, float v) const {
    if (ci >= s.Ci) return;
    int64_t u = q;
    const int iw = (int)(u % c.n[2]); u /= c.n[2];
    const int ih = (int)(u % c.n[1]); u /= c.n[1];
    const int id = (int)(u % c.n[0]);
    const int b = (int)(u / c.n[0]);
    const int d = 2 * id + c.p[0], h = 2 * ih + c.p[1], w = 2 * iw + c.p[2];
    dx[((((int64_t)b * s.D + d) * s.H + h) * s.W + w) * s.Ci + ci] = v;
  }
};

// ---------------------------------------------------------------------------
// launchers

template <class LA, class LB, class EP>
static void gemm_launch(int bn, LA la, LB lb, EP ep, int64_t rows, int64_t red, int64_t red_split,
                        int splits, cudaStream_t st) {
  const dim3 grid((unsigned)((rows + kBM - 1) / kBM), (unsigned)splits);
  switch (bn) {
    case 16: k_conv_gemm<16><<<grid, kConvThreads, 0, st>>>(la, lb, ep, rows, red, red_split); break;
    case 32: k_conv_gemm<32><<<grid, kConvThreads, 0, st>>>(la, lb, ep, rows, red, red_split); break;
    case 64: k_conv_gemm<64><<<grid, kConvThreads, 0, st>>>(la, lb, ep, rows, red, red_split); break;
    default: k_conv_gemm<128><<<grid, kConvThreads, 0, st>>>(la, lb, ep, rows, red, red_split); break;
  }
  count_launches(1);
}

static int pad_cols(int c) { return c <= 16 ? 16 : (c <= 32 ? 32 : (c <= 64 ? 64 : 128)); }

bool conv_shape(int B, int D, int H, int W, int Ci, int Co, ConvShape& s) {
  if (B <= 0 || D <= 0 || H <= 0 || W <= 0 || Ci <= 0 || Co <= 0 || Co > 128 || Ci > 128)
    return false;
  if (Co != 16 && Co != 32 && Co != 64 && Co != 128) return false;
  s.B = B; s.D = D; s.H = H; s.W = W; s.Ci = Ci; s.Co = Co;
  s.Do = (D + 1) / 2; s.Ho = (H + 1) / 2; s.Wo = (W + 1) / 2;
  s.K = 27 * Ci;
  s.Kp = (s.K + kBK - 1) / kBK * kBK;
  s.M = (int64_t)B * s.Do * s.Ho * s.Wo;
  return true;
}

static int wgrad_splits(const ConvShape& s) {
  const int64_t row_tiles = (s.Kp + kBM - 1) / kBM;
  int64_t sp = std::max<int64_t>(1, (int64_t)148 * 4 / row_tiles);
  sp = std::min<int64_t>(sp, std::max<int64_t>(1, s.M / (4 * kBK)));
  return (int)sp;
}

size_t conv_ws_bytes(const ConvShape& s) {
  const size_t dp = ((size_t)s.M * s.Co * sizeof(bf16) + 255) / 256 * 256;
  const size_t part = (size_t)wgrad_splits(s) * s.Kp * s.Co * sizeof(float);
  return dp + part + 256;
}

int launch_conv_forward(const ConvShape& s, const bf16* x, const bf16* w, const float* bias,
                        float* pre, bf16* act, cudaStream_t st) {
  gemm_launch(s.Co, FwdA{x, s}, WeightB{w, s.Co}, FwdEp{bias, pre, act, s.Co}, s.M, s.Kp, s.Kp,
              1, st);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

int launch_conv_backward(const ConvShape& s, const bf16* x, const bf16* w, const float* pre,
                         const float* dact, float* dx, float* dw, float* db, void* ws,
                         cudaStream_t st) {
  char* base = (char*)ws;
  bf16* dp = (bf16*)base;
  float* part = (float*)(base + ((size_t)s.M * s.Co * sizeof(bf16) + 255) / 256 * 256);
  const int64_t nout = s.M * s.Co;
  k_gelu_back<<<(unsigned)std::min<int64_t>((nout + 255) / 256, 148 * 16), 256, 0, st>>>(
      pre, dact, dp, nout);
  count_launches(1);
  // weight gradient: rows = Kp, reduction over m split across blockIdx.y
  const int splits = wgrad_splits(s);
  const int64_t per = ((s.M + splits - 1) / splits + kBK - 1) / kBK * kBK;
  const int used = (int)((s.M + per - 1) / per);
  gemm_launch(s.Co, WgradA{x, s}, DpreB{dp, s.Co}, WgradEp{part, (int64_t)s.Kp * s.Co, s.Co},
              (int64_t)s.Kp, s.M, per, used, st);
  const int64_t nw = (int64_t)s.Kp * s.Co;
  k_sum_splits<<<(unsigned)std::min<int64_t>((nw + 255) / 256, 148 * 4), 256, 0, st>>>(part, used,
                                                                                       nw, dw);
  k_bias_grad<<<s.Co, 256, 0, st>>>(dp, s.M, s.Co, db);
  count_launches(2);
  // data gradient: one GEMM per parity class of the input voxels
  if (dx) {
    for (int cls = 0; cls < 8; ++cls) {
      Cls c;
      const int dims[3] = {s.D, s.H, s.W};
      c.T = 1;
      bool empty = false;
      for (int a = 0; a < 3; ++a) {
        c.p[a] = (cls >> (2 - a)) & 1;
        c.n[a] = (dims[a] - c.p[a] + 1) / 2;
        c.nt[a] = c.p[a] == 0 ? 1 : 2;
        c.T *= c.nt[a];
        if (c.n[a] <= 0) empty = true;
      }
      if (empty) continue;
      const int64_t rows = (int64_t)s.B * c.n[0] * c.n[1] * c.n[2];
      const int64_t red = ((int64_t)c.T * s.Co + kBK - 1) / kBK * kBK;
      gemm_launch(pad_cols(s.Ci), DgradA{dp, s, c}, DgradB{w, s, c}, DgradEp{dx, s, c}, rows, red,
                  red, 1, st);
    }
  }
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

}  // namespace dm

// ---------------------------------------------------------------------------
extern "C" {

size_t dm_conv3d_s2_workspace_size(int B, int D, int H, int W, int Ci, int Co) {
  dm::ConvShape s;
  if (!dm::conv_shape(B, D, H, W, Ci, Co, s)) return 0;
  return dm::conv_ws_bytes(s);
}

int dm_conv3d_s2_forward(const uint16_t* x, int B, int D, int H, int W, int Ci, const uint16_t* w,
                         const float* bias, int Co, float* pre, uint16_t* act,
                         dm_stream_t stream) {
  dm::ConvShape s;
  if (!dm::conv_shape(B, D, H, W, Ci, Co, s)) return DM_ERR_INVALID_ARG;
  if (!x || !w || !pre || !act) return DM_ERR_INVALID_ARG;
  return dm::launch_conv_forward(s, (const dm::bf16*)x, (const dm::bf16*)w, bias, pre,
                                 (dm::bf16*)act, (cudaStream_t)stream);
}

int dm_conv3d_s2_backward(const uint16_t* x, int B, int D, int H, int W, int Ci,
                          const uint16_t* w, int Co, const float* pre, const float* dact,
                          float* dx, float* dw, float* db, void* workspace, size_t ws_bytes,
                          dm_stream_t stream) {
  dm::ConvShape s;
  if (!dm::conv_shape(B, D, H, W, Ci, Co, s)) return DM_ERR_INVALID_ARG;
  if (!x || !w || !pre || !dact || !dw || !db || !workspace) return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm::conv_ws_bytes(s)) return DM_ERR_WORKSPACE;
  return dm::launch_conv_backward(s, (const dm::bf16*)x, (const dm::bf16*)w, pre, dact, dx, dw, db,
                                  workspace, (cudaStream_t)stream);
}

}  // extern "C"
