// Segmentation masks of deltamic/mask_creation.py on the GPU.
//
//  * Membrane ("semantic") mask, create_semantic_segmentation_mask
//    (mask_creation.py:208-222): the mesh is refined until every edge is at most
//    one voxel (trimesh's subdivide_to_size: faces with a longer edge split four
//    ways at their edge midpoints (a + b) / 2), and the grid point nearest to every
//    vertex of the refined mesh is set to 1.  One thread refines one face depth
//    first, so no refined mesh is ever stored; the grid points are
//    numpy.linspace(lo, hi, n) per axis (create_coords, :195-205), whose nearest
//    point is found per axis.
//  * Label ("instance") mask, create_instance_segmentation_mask (:225-266): faces
//    carry the labels of the regions on either side; every face is split four ways
//    `levels` times (subdivide_with_materials, :60-176), and every grid point takes
//    the label on its side of the nearest child face (nearest centroid, side by the
//    sign of (centroid - point) . normal), plus one.  The nearest centroid is an
//    exhaustive search over centroid tiles staged in shared memory (exact; ties go
//    to the lower child index).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/deltamic_b200.h"
#include "dm_common.cuh"
#include "meshft_internal.h"

namespace dm {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxDepth = 24;     // refinement levels of the membrane mask
constexpr int kTile = 256;        // centroids per shared-memory tile

int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }
int status() { return cudaGetLastError() == cudaSuccess ? DM_OK : DM_ERR_CUDA; }

struct Axes {
  double lo[3], hi[3], step[3];
  int32_t n[3];
};

Axes make_axes(const dm_box* b) {
  Axes a;
  for (int d = 0; d < 3; ++d) {
    a.lo[d] = b->lo[d];
    a.hi[d] = b->hi[d];
    a.n[d] = b->shape[d];
    a.step[d] = b->shape[d] > 1 ? (b->hi[d] - b->lo[d]) / (b->shape[d] - 1) : 0.0;
  }
  return a;
}

// numpy.linspace(lo, hi, n)[i]: i * step + lo, the last point exactly hi.
__device__ __forceinline__ double grid_value(const Axes& a, int d, int i) {
  return i == a.n[d] - 1 ? a.hi[d] : __dadd_rn(__dmul_rn((double)i, a.step[d]), a.lo[d]);
}

// Index of the grid value nearest to x along axis d (the lower one on a tie).
__device__ __forceinline__ int nearest_index(const Axes& a, int d, double x) {
  const int n = a.n[d];
  if (n == 1) return 0;
  const double t = (x - a.lo[d]) / a.step[d];
  int i = isfinite(t) ? (int)fmin(fmax(floor(t), 0.0), (double)(n - 1)) : 0;
  int best = -1;
  double bd = 0.0;
  for (int c = i - 1; c <= i + 2; ++c) {
    if (c < 0 || c >= n) continue;
    const double dist = fabs(x - grid_value(a, d, c));
    if (best < 0 || dist < bd) {
      best = c;
      bd = dist;
    }
  }
  return best;
}

struct Tri {
  double p[3][3];
  int depth;
};

__device__ __forceinline__ double edge_len(const double* u, const double* v) {
  const double dx = v[0] - u[0], dy = v[1] - u[1], dz = v[2] - u[2];
  return sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
}

__device__ __forceinline__ void midpoint(const double* u, const double* v, double* m) {
#pragma unroll
  for (int j = 0; j < 3; ++j) m[j] = (u[j] + v[j]) / 2.0;
}

// Child c (0..3) of triangle (a, b, c) in trimesh's order:
// (a, ab, ca), (ab, b, bc), (ca, bc, c), (ab, bc, ca).
__device__ __forceinline__ void child(const double (&t)[3][3], int c, double (&o)[3][3]) {
  double ab[3], bc[3], ca[3];
  midpoint(t[0], t[1], ab);
  midpoint(t[1], t[2], bc);
  midpoint(t[2], t[0], ca);
  const double* q[4][3] = {{t[0], ab, ca}, {ab, t[1], bc}, {ca, bc, t[2]}, {ab, bc, ca}};
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int j = 0; j < 3; ++j) o[k][j] = q[c][k][j];
}

// One thread per face: depth-first refinement, the nearest grid point of every
// vertex of every final triangle set to 1 (racing writes store the same value).
__global__ void k_membrane(const double* __restrict__ verts, int64_t nv,
                           const int64_t* __restrict__ faces, int fstride, int64_t nt,
                           double max_edge, int max_depth, Axes a, double* __restrict__ mask,
                           int* err) {
  const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nt) return;
  Tri stack[3 * kMaxDepth + 4];
  int top = 0;
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int64_t v = faces[f * fstride + k];
    if (v < 0 || v >= nv) ok = false;
#pragma unroll
    for (int j = 0; j < 3; ++j) stack[0].p[k][j] = ok ? verts[3 * v + j] : 0.0;
  }
  if (!ok) {
    set_error(err, DM_ERR_BAD_INDEX);
    return;
  }
  stack[0].depth = 0;
  top = 1;
  const int64_t nyz = (int64_t)a.n[1] * a.n[2];
  while (top > 0) {
    const Tri t = stack[--top];
    const double e = fmax(fmax(edge_len(t.p[0], t.p[1]), edge_len(t.p[1], t.p[2])),
                          edge_len(t.p[2], t.p[0]));
    if (e > max_edge) {
      if (t.depth >= max_depth) {  // trimesh raises "max_iter exceeded"
        set_error(err, DM_ERR_SIZE);
        return;
      }
      for (int c = 3; c >= 0; --c) {
        child(t.p, c, stack[top].p);
        stack[top].depth = t.depth + 1;
        ++top;
      }
      continue;
    }
    for (int k = 0; k < 3; ++k) {
      const int ix = nearest_index(a, 0, t.p[k][0]);
      const int iy = nearest_index(a, 1, t.p[k][1]);
      const int iz = nearest_index(a, 2, t.p[k][2]);
      mask[(int64_t)ix * nyz + (int64_t)iy * a.n[2] + iz] = 1.0;
    }
  }
}

// Children of every face after `levels` four-way splits, in the reference's order
// (child index = face * 4^levels + digits, most significant first): centroid,
// unit normal (b - a) x (c - b), and the labels, the larger first (reorder_faces,
// mask_creation.py:49-53: a face whose first label is the smaller one is flipped).
__global__ void k_children(const double* __restrict__ verts, int64_t nv,
                           const int64_t* __restrict__ faces, int64_t nt, int levels,
                           double* __restrict__ cen, double* __restrict__ nrm,
                           double* __restrict__ lab, int* err) {
  const int64_t per = (int64_t)1 << (2 * levels);
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt * per) return;
  const int64_t f = i / per;
  const int64_t digits = i - f * per;
  int64_t v[3];
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    v[k] = faces[5 * f + k];
    if (v[k] < 0 || v[k] >= nv) ok = false;
  }
  if (!ok) {
    set_error(err, DM_ERR_BAD_INDEX);
    return;
  }
  int64_t l1 = faces[5 * f + 3], l2 = faces[5 * f + 4];
  if (l1 < l2) {  // [0, 2, 1, 4, 3]
    const int64_t s = v[1];
    v[1] = v[2];
    v[2] = s;
    const int64_t sl = l1;
    l1 = l2;
    l2 = sl;
  }
  double t[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int j = 0; j < 3; ++j) t[k][j] = verts[3 * v[k] + j];
  for (int lv = levels - 1; lv >= 0; --lv) {
    double o[3][3];
    child(t, (int)((digits >> (2 * lv)) & 3), o);
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int j = 0; j < 3; ++j) t[k][j] = o[k][j];
  }
  double T1[3], T2[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    cen[3 * i + j] = (t[0][j] + t[1][j] + t[2][j]) / 3.0;
    T1[j] = t[1][j] - t[0][j];
    T2[j] = t[2][j] - t[1][j];
  }
  const double n0 = __dsub_rn(__dmul_rn(T1[1], T2[2]), __dmul_rn(T1[2], T2[1]));
  const double n1 = __dsub_rn(__dmul_rn(T1[2], T2[0]), __dmul_rn(T1[0], T2[2]));
  const double n2 = __dsub_rn(__dmul_rn(T1[0], T2[1]), __dmul_rn(T1[1], T2[0]));
  const double nn = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(n0, n0), __dmul_rn(n1, n1)),
                                   __dmul_rn(n2, n2)));
  nrm[3 * i + 0] = n0 / nn;
  nrm[3 * i + 1] = n1 / nn;
  nrm[3 * i + 2] = n2 / nn;
  lab[2 * i + 0] = (double)l1;
  lab[2 * i + 1] = (double)l2;
}

// One thread per grid point: nearest centroid over all children (tiles in shared
// memory, lower index on ties), then the label on the point's side of its normal.
__global__ void __launch_bounds__(kThreads)
    k_nearest_label(const double* __restrict__ cen, const double* __restrict__ nrm,
                    const double* __restrict__ lab, int64_t nc, Axes a,
                    double* __restrict__ out) {
  __shared__ double sc[kTile][3];
  const int64_t npts = (int64_t)a.n[0] * a.n[1] * a.n[2];
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = p < npts;
  double q[3] = {0.0, 0.0, 0.0};
  if (live) {
    const int64_t nyz = (int64_t)a.n[1] * a.n[2];
    const int ix = (int)(p / nyz), iy = (int)((p / a.n[2]) % a.n[1]), iz = (int)(p % a.n[2]);
    q[0] = grid_value(a, 0, ix);
    q[1] = grid_value(a, 1, iy);
    q[2] = grid_value(a, 2, iz);
  }
  double best = INFINITY;
  int64_t bi = 0;
  for (int64_t t0 = 0; t0 < nc; t0 += kTile) {
    const int cnt = (int)(nc - t0 < kTile ? nc - t0 : kTile);
    __syncthreads();
    for (int k = threadIdx.x; k < cnt * 3; k += blockDim.x) sc[k / 3][k % 3] = cen[3 * t0 + k];
    __syncthreads();
    for (int k = 0; k < cnt; ++k) {
      const double dx = sc[k][0] - q[0], dy = sc[k][1] - q[1], dz = sc[k][2] - q[2];
      const double d = dx * dx + dy * dy + dz * dz;
      if (d < best) {
        best = d;
        bi = t0 + k;
      }
    }
  }
  if (!live) return;
  const double vx = cen[3 * bi] - q[0], vy = cen[3 * bi + 1] - q[1], vz = cen[3 * bi + 2] - q[2];
  const double dot = __dadd_rn(__dadd_rn(__dmul_rn(vx, nrm[3 * bi]), __dmul_rn(vy, nrm[3 * bi + 1])),
                               __dmul_rn(vz, nrm[3 * bi + 2]));
  out[p] = lab[2 * bi + (dot < 0.0 ? 1 : 0)] + 1.0;
}

bool box_fine(const dm_box* b) {
  if (!b) return false;
  for (int d = 0; d < 3; ++d)
    if (b->shape[d] <= 0 || (b->shape[d] > 1 && !(b->hi[d] > b->lo[d]))) return false;
  return (int64_t)b->shape[0] * b->shape[1] * b->shape[2] <= ((int64_t)1 << 40);
}

}  // namespace
}  // namespace dm

using namespace dm;

extern "C" {

size_t dm_mask_workspace_size(int64_t nt, int32_t levels) {
  if (nt < 0 || levels < 0 || levels > 8) return 0;
  const int64_t nc = nt << (2 * levels);
  return 256 + sizeof(double) * 8 * (size_t)std::max<int64_t>(nc, 1);
}

int dm_membrane_mask(const double* verts, int64_t nv, const int64_t* faces, int64_t nt,
                     int32_t face_stride, const dm_box* box, double max_edge, int32_t max_depth,
                     double* mask, void* workspace, size_t ws_bytes, dm_stream_t stream) {
  if (!box_fine(box) || !mask || !workspace || nv < 0 || nt < 0 || face_stride < 3 ||
      (nt > 0 && (!verts || !faces)) || !(max_edge > 0.0))
    return DM_ERR_INVALID_ARG;
  if (max_depth < 0 || max_depth > kMaxDepth) return DM_ERR_SIZE;
  if (ws_bytes < 256) return DM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t npts = (int64_t)box->shape[0] * box->shape[1] * box->shape[2];
  if (cudaMemsetAsync(mask, 0, sizeof(double) * (size_t)npts, st) != cudaSuccess)
    return DM_ERR_CUDA;
  if (nt == 0) return DM_OK;
  k_membrane<<<(unsigned)cdiv(nt, 128), 128, 0, st>>>(verts, nv, faces, face_stride, nt,
                                                       max_edge, max_depth, make_axes(box), mask,
                                                       (int*)workspace);
  count_launches(1);
  return status();
}

int dm_instance_mask(const double* verts, int64_t nv, const int64_t* faces, int64_t nt,
                     const dm_box* box, int32_t levels, double* mask, void* workspace,
                     size_t ws_bytes, dm_stream_t stream) {
  if (!box_fine(box) || !mask || !workspace || nv < 0 || nt <= 0 || !verts || !faces ||
      levels < 0 || levels > 8)
    return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm_mask_workspace_size(nt, levels)) return DM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t nc = nt << (2 * levels);
  char* w = (char*)workspace;
  int* err = (int*)w;
  double* cen = (double*)(w + 256);
  double* nrm = cen + 3 * nc;
  double* lab = nrm + 3 * nc;
  k_children<<<(unsigned)cdiv(nc, kThreads), kThreads, 0, st>>>(verts, nv, faces, nt, levels,
                                                                 cen, nrm, lab, err);
  const int64_t npts = (int64_t)box->shape[0] * box->shape[1] * box->shape[2];
  k_nearest_label<<<(unsigned)cdiv(npts, kThreads), kThreads, 0, st>>>(cen, nrm, lab, nc,
                                                                        make_axes(box), mask);
  count_launches(2);
  return status();
}

}  // extern "C"
