// Throughput probes used as roofline denominators: FP32 FMA and MUFU sine
// (sin.approx.f32) issue rates of this GPU, measured with independent chains.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/deltamic_b200.h"
#include "dm_common.cuh"

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

// Paired FP32 FMA (sm_100 FFMA2: two fused multiply-adds per instruction).
__global__ void k_peak_ffma2(int iters, float a, float b) {
  float2 x[kChains];
  const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = make_float2(threadIdx.x * 1e-3f + c, c * 0.5f);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = __ffma2_rn(x[c], a2, b2);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c].x + x[c].y;
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

// Self-test of the bounded waits: an mbarrier that nothing arrives on (no copy is
// issued, so none is in flight); every thread polls it at most ``limit`` times
// with the kernels' spinning (mode 0) or sleeping (mode 1) wait, gives up, sets
// DM_ERR_TIMEOUT in *err and returns.
__global__ void k_wait_selftest(int mode, uint32_t limit, int* err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  const bool ok = mode == 0 ? mbar_wait_bounded(&bar, 0, err, limit)
                            : mbar_wait_sleep_bounded(&bar, 0, err, limit);
  if (ok) atomicOr(err, DM_ERR_INVALID_ARG);  // the phase can never complete
}

}  // namespace dm

extern "C" int dm_selftest_bounded_wait(int mode, uint32_t limit, int* status,
                                        dm_stream_t stream) {
  if ((mode != 0 && mode != 1) || !status || limit == 0) return DM_ERR_INVALID_ARG;
  if (limit > (mode == 0 ? dm::kWaitLimit : dm::kSleepTries)) return DM_ERR_SIZE;
  dm::k_wait_selftest<<<1, 64, 0, (cudaStream_t)stream>>>(mode, limit, status);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

extern "C" int dm_peak_probe(int kind, int iters, double* ops_per_s, dm_stream_t stream) {
  if (kind < 0 || kind > 2 || iters <= 0 || !ops_per_s) return DM_ERR_INVALID_ARG;
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
    else if (kind == 1)
      dm::k_peak_mufu<<<blocks, threads, 0, st>>>(iters);
    else
      dm::k_peak_ffma2<<<blocks, threads, 0, st>>>(iters, 0.999f, 1e-3f);
  }
  cudaEventRecord(e1, st);
  int status = cudaEventSynchronize(e1) == cudaSuccess ? DM_OK : DM_ERR_CUDA;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // FMAs (kinds 0 and 2: an FFMA2 is two) or sines per second
  const double ops = (double)blocks * threads * iters * dm::kChains * (kind == 2 ? 2 : 1);
  *ops_per_s = ms > 0.f ? ops / (ms * 1e-3) : 0.0;
  return status;
}
