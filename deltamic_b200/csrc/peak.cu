// Throughput probes used as roofline denominators: FP32 FMA and MUFU sine
// (sin.approx.f32) issue rates of this GPU, measured with independent chains.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/deltamic_b200.h"

namespace dm {

constexpr int kChains = 8;
__device__ float g_peak_sink;  // keeps the chains alive without a caller buffer

__global__ void k_peak_fma(int iters, float a, float b) {
  float x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-3f + c;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = fmaf(x[c], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  if (s == 12345.678f) g_peak_sink = s;
}

__global__ void k_peak_mufu(int iters) {
  float x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-3f + 0.1f * c;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) asm volatile("sin.approx.ftz.f32 %0, %0;" : "+f"(x[c]));
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  if (s == 12345.678f) g_peak_sink = s;
}

}  // namespace dm

extern "C" int dm_peak_probe(int kind, int iters, double* ops_per_s, dm_stream_t stream) {
  if ((kind != 0 && kind != 1) || iters <= 0 || !ops_per_s) return DM_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int threads = 256, blocks = sms * 8;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // warm-up, then timed launch
  for (int rep = 0; rep < 2; ++rep) {
    if (rep == 1) cudaEventRecord(e0, st);
    if (kind == 0)
      dm::k_peak_fma<<<blocks, threads, 0, st>>>(iters, 0.999f, 1e-3f);
    else
      dm::k_peak_mufu<<<blocks, threads, 0, st>>>(iters);
  }
  cudaEventRecord(e1, st);
  int status = cudaEventSynchronize(e1) == cudaSuccess ? DM_OK : DM_ERR_CUDA;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const double ops = (double)blocks * threads * iters * dm::kChains;
  *ops_per_s = ms > 0.f ? ops / (ms * 1e-3) : 0.0;
  return status;
}
