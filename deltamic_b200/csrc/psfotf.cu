// OTF of a spatial PSF: OTF = |fftshift(fftn(PSF))| (the notebook's
// `OTF = torch.abs(torch.fft.fftshift(torch.fft.fftn(PSF)))`,
// Examples/Gradient_Descent.ipynb cell 2, with PSF from psf.py:551-587) and its
// adjoint.  The 3-D transform itself is cuFFT's (through torch.fft); these kernels
// fuse the shift with |.| and, backward, the unshift with d|F|/dF = F/|F|.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "band_internal.h"
#include "dm_common.cuh"

namespace dm {
namespace {

// out[k] = |F[(k - n/2) mod n]| per axis (fftshift moves index 0 to n/2).
__global__ void k_shift_abs(const float2* __restrict__ F, int32_t n0, int32_t n1, int32_t n2,
                            float* __restrict__ otf) {
  const int64_t nvox = (int64_t)n0 * n1 * n2;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nvox;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t k0 = (int32_t)(k / ((int64_t)n1 * n2));
    const int32_t r = (int32_t)(k - (int64_t)k0 * n1 * n2);
    const int32_t k1 = r / n2, k2 = r - k1 * n2;
    const int32_t j0 = (k0 + n0 - n0 / 2) % n0, j1 = (k1 + n1 - n1 / 2) % n1;
    const int32_t j2 = (k2 + n2 - n2 / 2) % n2;
    const float2 f = F[((int64_t)j0 * n1 + j1) * n2 + j2];
    otf[k] = sqrtf(fmaf(f.x, f.x, f.y * f.y));
  }
}

// gF[j] = g[(j + n/2) mod n] * F[j] / |F[j]| (0 where F[j] = 0), PyTorch's complex
// convention for the gradient of |.|.
__global__ void k_shift_abs_bwd(const float2* __restrict__ F, const float* __restrict__ g,
                                int32_t n0, int32_t n1, int32_t n2, float2* __restrict__ gF) {
  const int64_t nvox = (int64_t)n0 * n1 * n2;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nvox;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int32_t j0 = (int32_t)(j / ((int64_t)n1 * n2));
    const int32_t r = (int32_t)(j - (int64_t)j0 * n1 * n2);
    const int32_t j1 = r / n2, j2 = r - j1 * n2;
    const int32_t k0 = (j0 + n0 / 2) % n0, k1 = (j1 + n1 / 2) % n1, k2 = (j2 + n2 / 2) % n2;
    const float gk = g[((int64_t)k0 * n1 + k1) * n2 + k2];
    const float2 f = F[j];
    const float a = sqrtf(fmaf(f.x, f.x, f.y * f.y));
    const float sc = a > 0.f ? gk / a : 0.f;
    gF[j] = make_float2(sc * f.x, sc * f.y);
  }
}

unsigned grid_for(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return (unsigned)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

}  // namespace
}  // namespace dm

using namespace dm;

extern "C" {

int dm_otf_from_spectrum(const float* spectrum, int32_t n0, int32_t n1, int32_t n2, float* otf,
                         dm_stream_t stream) {
  if (!spectrum || !otf || n0 <= 0 || n1 <= 0 || n2 <= 0) return DM_ERR_INVALID_ARG;
  const int64_t n = (int64_t)n0 * n1 * n2;
  if (n > (int64_t)INT32_MAX) return DM_ERR_SIZE;
  k_shift_abs<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((const float2*)spectrum, n0, n1, n2,
                                                              otf);
  count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

int dm_otf_from_spectrum_backward(const float* spectrum, const float* grad_otf, int32_t n0,
                                  int32_t n1, int32_t n2, float* grad_spectrum,
                                  dm_stream_t stream) {
  if (!spectrum || !grad_otf || !grad_spectrum || n0 <= 0 || n1 <= 0 || n2 <= 0)
    return DM_ERR_INVALID_ARG;
  const int64_t n = (int64_t)n0 * n1 * n2;
  if (n > (int64_t)INT32_MAX) return DM_ERR_SIZE;
  k_shift_abs_bwd<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(
      (const float2*)spectrum, grad_otf, n0, n1, n2, (float2*)grad_spectrum);
  count_launches(1);
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

}  // extern "C"
