// Internal launch interface of the narrow-band, OTF and image kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/deltamic_b200.h"
#include "dm_common.cuh"

namespace dm {

void count_launches(int n);

int64_t band_blocks(int64_t n);
int launch_narrowband(const float* otf, int64_t n, float thresh, int32_t* out, int64_t* count,
                      int32_t* blk_count, int32_t* blk_off, cudaStream_t st);
int launch_narrowband64(const double* otf, int64_t n, double thresh, int32_t* out,
                        int64_t* count, int32_t* blk_count, int32_t* blk_off, cudaStream_t st);
int launch_band_mirror(const int32_t* band, int64_t nb, int64_t nvox, int32_t* flag,
                       cudaStream_t st);
int launch_gaussian_otf(const float* sigma, const float* const xi[3], const int32_t n[3],
                        float* otf, cudaStream_t st);
int launch_gaussian_otf64(const double* sigma, const double* const xi[3], const int32_t n[3],
                          double* otf, cudaStream_t st);
int otf_grad_blocks(int64_t n);
int launch_otf_sigma_grad64(const double* gotf, const int32_t* band, int64_t n,
                            const double* otf, const double* const xi[3], const int32_t nax[3],
                            double* grad_sigma, double* part, cudaStream_t st);
int launch_otf_sigma_grad(const float* gotf, const int32_t* band, int64_t n, const float* otf,
                          const float* const xi[3], const int32_t nax[3], float* grad_sigma,
                          double* part, cudaStream_t st);

// image stage
struct ImgStats {
  float mn, mx;
  int64_t imn, imx;
};
constexpr int kTieSlots = 1024;
int image_blocks(int64_t n);
size_t image_ws_bytes(int64_t n);
size_t image_ws_bytes_segs(int64_t max_len, int nseg);
int launch_image_loss(const float2* z, int64_t n, int kind, const float* target, float contrast,
                      float* image, float* loss, float2* grad_z, void* ws, cudaStream_t st);
int launch_image_loss_cells(const CellDesc* cells, int ncells, int64_t max_len, const float2* z,
                            int kind, const float* target, float contrast, float* image,
                            float* loss, float2* grad_z, void* ws, cudaStream_t st);
int launch_voxelize(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                    const dm_box& box, uint8_t* occ, int* err, cudaStream_t st);
int launch_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1,
                float b2, float eps, int64_t* step, cudaStream_t st);

}  // namespace dm
