// Occupancy of a closed triangle mesh on a box grid, for the volumetric IoU of
// fitted meshes (evaluation of the fitting loop).  One thread per z-column:
// every triangle whose xy projection contains the column's (x, y) contributes a
// crossing height; a voxel is inside when an odd number of crossings lie below
// it.  Triangles are staged in shared memory tiles read by the whole block.
// Voxel (i, j, k) sits at lo + (i, j, k) * L / n, the sample positions of the
// rendered image (abs(ifftn) of the centred spectrum).
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/deltamic_b200.h"
#include "band_internal.h"

namespace dm {

constexpr int kVoxThreads = 128;
constexpr int kVoxTile = 128;
constexpr int kMaxCross = 64;

struct Tri2 {
  double ax, ay, az, bx, by, bz, cx, cy, cz;
};

__global__ void k_voxelize(const float* __restrict__ verts, int64_t nv,
                           const int64_t* __restrict__ faces, int64_t nt, dm_box box,
                           uint8_t* __restrict__ occ, int* err) {
  __shared__ Tri2 tile[kVoxTile];
  const int n0 = box.shape[0], n1 = box.shape[1], n2 = box.shape[2];
  const int64_t col = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = col < (int64_t)n0 * n1;
  const int i = active ? (int)(col / n1) : 0, j = active ? (int)(col % n1) : 0;
  const double L0 = box.hi[0] - box.lo[0], L1 = box.hi[1] - box.lo[1];
  // small irrational offsets keep columns off shared edges and vertices
  const double px = box.lo[0] + (i + 0.3819660113e-6) * L0 / n0;
  const double py = box.lo[1] + (j + 0.6180339887e-6) * L1 / n1;
  double zc[kMaxCross];
  int nc = 0;
  for (int64_t t0 = 0; t0 < nt; t0 += kVoxTile) {
    __syncthreads();
    for (int t = threadIdx.x; t < kVoxTile && t0 + t < nt; t += blockDim.x) {
      const int64_t f = t0 + t;
      int64_t ia = faces[3 * f], ib = faces[3 * f + 1], ic = faces[3 * f + 2];
      if (ia < 0 || ia >= nv || ib < 0 || ib >= nv || ic < 0 || ic >= nv) {
        if (err) atomicOr(err, DM_ERR_BAD_INDEX);
        ia = ib = ic = 0;
      }
      Tri2 r;
      r.ax = verts[3 * ia]; r.ay = verts[3 * ia + 1]; r.az = verts[3 * ia + 2];
      r.bx = verts[3 * ib]; r.by = verts[3 * ib + 1]; r.bz = verts[3 * ib + 2];
      r.cx = verts[3 * ic]; r.cy = verts[3 * ic + 1]; r.cz = verts[3 * ic + 2];
      tile[t] = r;
    }
    __syncthreads();
    const int m = (int)(nt - t0 < kVoxTile ? nt - t0 : kVoxTile);
    if (!active) continue;
    for (int t = 0; t < m; ++t) {
      const Tri2 r = tile[t];
      const double d = (r.bx - r.ax) * (r.cy - r.ay) - (r.cx - r.ax) * (r.by - r.ay);
      if (d == 0.0) continue;
      const double w1 = ((px - r.ax) * (r.cy - r.ay) - (r.cx - r.ax) * (py - r.ay)) / d;
      const double w2 = ((r.bx - r.ax) * (py - r.ay) - (px - r.ax) * (r.by - r.ay)) / d;
      const double w0 = 1.0 - w1 - w2;
      if (w0 < 0.0 || w1 < 0.0 || w2 < 0.0) continue;
      if (nc < kMaxCross) {
        zc[nc++] = w0 * r.az + w1 * r.bz + w2 * r.cz;
      } else if (err) {
        atomicOr(err, DM_ERR_SIZE);
      }
    }
  }
  if (!active) return;
  for (int a = 1; a < nc; ++a) {  // insertion sort of the crossings
    const double x = zc[a];
    int b = a - 1;
    while (b >= 0 && zc[b] > x) {
      zc[b + 1] = zc[b];
      --b;
    }
    zc[b + 1] = x;
  }
  const double L2 = box.hi[2] - box.lo[2];
  int below = 0;
  uint8_t* out = occ + ((int64_t)i * n1 + j) * n2;
  for (int k = 0; k < n2; ++k) {
    const double z = box.lo[2] + k * L2 / n2;
    while (below < nc && zc[below] < z) ++below;
    out[k] = (uint8_t)(below & 1);
  }
}

int launch_voxelize(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                    const dm_box& box, uint8_t* occ, int* err, cudaStream_t st) {
  const int64_t cols = (int64_t)box.shape[0] * box.shape[1];
  const int64_t blocks = (cols + kVoxThreads - 1) / kVoxThreads;
  if (blocks > 0) {
    k_voxelize<<<(unsigned)blocks, kVoxThreads, 0, st>>>(verts, nv, faces, nt, box, occ, err);
    count_launches(1);
  }
  return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA;
}

}  // namespace dm
