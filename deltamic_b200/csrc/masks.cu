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
//    sign of (centroid - point) . normal), plus one.  The nearest centroid is exact
//    (ties go to the lower child index): the centroids are counting-sorted into a
//    uniform grid of buckets with tight bounding boxes; each point first bounds its
//    nearest distance by the farthest corner of every non-empty bucket, then reads
//    the centroids of the buckets whose nearest corner is within that bound.
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

// Uniform bucket grid over the query box (centroids outside it go to the border
// buckets; every bucket's box is the tight box of its own centroids).
struct Buckets {
  double lo[3], inv[3], h[3];  // h = 1 / inv: the bucket edge
  int32_t n[3];
};

__device__ __forceinline__ int64_t bucket_of(const Buckets& g, const double* c) {
  int64_t idx = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double t = (c[d] - g.lo[d]) * g.inv[d];
    const int i = isfinite(t) ? (int)fmin(fmax(floor(t), 0.0), (double)(g.n[d] - 1)) : 0;
    idx = idx * g.n[d] + i;
  }
  return idx;
}

__global__ void k_bucket_count(const double* __restrict__ cen, int64_t nc, Buckets g,
                               int32_t* __restrict__ count) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nc) atomicAdd(&count[bucket_of(g, cen + 3 * i)], 1);
}

// Exclusive scan of cnt[0..n) into off[0..n] by one block of 1024 threads
// (flags: the counts are turned into 0/1 first).
__global__ void k_scan(const int32_t* __restrict__ cnt, int64_t n, int flags,
                       int32_t* __restrict__ off) {
  __shared__ int32_t sh[1024];
  const int T = blockDim.x;
  const int64_t per = (n + T - 1) / T;
  const int64_t b = threadIdx.x * per, e = b + per < n ? b + per : n;
  int32_t s = 0;
  for (int64_t i = b; i < e; ++i) s += flags ? (cnt[i] > 0) : cnt[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < T; o <<= 1) {
    const int32_t v = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += v;
    __syncthreads();
  }
  int32_t run = sh[threadIdx.x] - s;
  for (int64_t i = b; i < e; ++i) {
    off[i] = run;
    run += flags ? (cnt[i] > 0) : cnt[i];
  }
  if (threadIdx.x == T - 1) off[n] = sh[T - 1];
}

__global__ void k_bucket_fill(const double* __restrict__ cen, int64_t nc, Buckets g,
                              const int32_t* __restrict__ off, int32_t* __restrict__ cursor,
                              int32_t* __restrict__ slot) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nc) return;
  const int64_t b = bucket_of(g, cen + 3 * i);
  slot[off[b] + atomicAdd(&cursor[b], 1)] = (int32_t)i;
}

// Non-empty buckets, in bucket order: tight box, first slot and count.
struct BucketRec {
  double lo[3], hi[3];
  int32_t first, count;
};

__global__ void k_bucket_boxes(const int32_t* __restrict__ off, const int32_t* __restrict__ nz_off,
                               const int32_t* __restrict__ slot, const double* __restrict__ cen,
                               int64_t nb, BucketRec* __restrict__ rec) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const int32_t s0 = off[b], s1 = off[b + 1];
  if (s1 == s0) return;
  BucketRec r;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    r.lo[d] = INFINITY;
    r.hi[d] = -INFINITY;
  }
  for (int32_t s = s0; s < s1; ++s) {
    const double* c = cen + 3 * (int64_t)slot[s];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      r.lo[d] = fmin(r.lo[d], c[d]);
      r.hi[d] = fmax(r.hi[d], c[d]);
    }
  }
  r.first = s0;
  r.count = s1 - s0;
  rec[nz_off[b]] = r;
}

constexpr double kSlackLabel = 1.0 + 1e-12;  // rounding of the box and face distances

__device__ __forceinline__ int bucket_axis(const Buckets& g, int d, double x) {
  const double t = (x - g.lo[d]) * g.inv[d];
  return isfinite(t) ? (int)fmin(fmax(floor(t), 0.0), (double)(g.n[d] - 1)) : 0;
}

// Distance from x to the faces of the visited cube (buckets c - r .. c + r on axis
// d) that have buckets beyond them, less a rounding margin (negative while x lies
// outside the cube).
__device__ __forceinline__ void face_bound(const Buckets& g, int d, int c, int r, double x,
                                           double& bound, bool& covered) {
  const double h = g.h[d];
  if (c - r > 0) {
    covered = false;
    bound = fmin(bound, x - (g.lo[d] + (c - r) * h) - 1e-9 * h);
  }
  if (c + r < g.n[d] - 1) {
    covered = false;
    bound = fmin(bound, (g.lo[d] + (c + r + 1) * h) - x - 1e-9 * h);
  }
}

// Grid points by warp: a warp takes a 2 x 4 x 4 brick of grid points (x, y, z),
// all of which usually fall in one bucket, and walks shells of buckets (Chebyshev
// distance r = 0, 1, 2, ... from the bucket of the brick's first point) together:
// a bucket is scanned when its tight box is within the best distance so far of
// any lane, every lane then measuring every centroid of it (no divergence), and
// the walk ends when every lane is done -- the nearest face of the visited cube
// with buckets beyond it is farther than that lane's best distance (every
// unvisited centroid lies beyond such a face: a centroid clamped into a border
// bucket lies beyond the box, hence beyond that face too), or the cube covers the
// grid.  The result per point is the exact nearest child centroid by (distance,
// child index); then the label on the point's side of that child.
constexpr int kBrickX = 2, kBrickY = 4, kBrickZ = 4;
__global__ void __launch_bounds__(kThreads)
    k_nearest_label(const double* __restrict__ cen, const double* __restrict__ nrm,
                    const double* __restrict__ lab, const int32_t* __restrict__ slot,
                    const int32_t* __restrict__ off, const int32_t* __restrict__ nzo,
                    const BucketRec* __restrict__ rec, Buckets g, Axes a,
                    double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nbx = (a.n[0] + kBrickX - 1) / kBrickX, nby = (a.n[1] + kBrickY - 1) / kBrickY,
            nbz = (a.n[2] + kBrickZ - 1) / kBrickZ;
  if (w >= (int64_t)nbx * nby * nbz) return;  // whole warp
  const int bz = (int)(w % nbz), by = (int)((w / nbz) % nby), bx = (int)(w / ((int64_t)nbz * nby));
  const int ix = bx * kBrickX + (lane >> 4), iy = by * kBrickY + ((lane >> 2) & 3),
            iz = bz * kBrickZ + (lane & 3);
  const bool live = ix < a.n[0] && iy < a.n[1] && iz < a.n[2];
  // lanes past the grid measure the brick's first point and store nothing
  const double q0 = grid_value(a, 0, live ? ix : bx * kBrickX);
  const double q1 = grid_value(a, 1, live ? iy : by * kBrickY);
  const double q2 = grid_value(a, 2, live ? iz : bz * kBrickZ);
  const int c0 = __shfl_sync(0xffffffffu, bucket_axis(g, 0, q0), 0);
  const int c1 = __shfl_sync(0xffffffffu, bucket_axis(g, 1, q1), 0);
  const int c2 = __shfl_sync(0xffffffffu, bucket_axis(g, 2, q2), 0);
  double best = INFINITY;
  int64_t bi = 0;
  const int rmax = max(g.n[0], max(g.n[1], g.n[2]));
  for (int r = 0; r <= rmax; ++r) {
    for (int dx = -r; dx <= r; ++dx) {
      const int x = c0 + dx;
      if (x < 0 || x >= g.n[0]) continue;
      const bool ex = dx == -r || dx == r;
      for (int dy = -r; dy <= r; ++dy) {
        const int y = c1 + dy;
        if (y < 0 || y >= g.n[1]) continue;
        const int64_t row = ((int64_t)x * g.n[1] + y) * g.n[2];
        // on an x or y face of the shell the whole z range, else its two z faces
        const int step = (ex || dy == -r || dy == r) ? 1 : 2 * r;
        for (int z = c2 - r; z <= c2 + r; z += step) {
          if (z < 0 || z >= g.n[2]) continue;
          const int64_t b = row + z;
          const int32_t s0 = off[b], s1 = off[b + 1];
          if (s0 == s1) continue;
          const BucketRec& rb = rec[nzo[b]];
          const double e0 = fmax(fmax(rb.lo[0] - q0, q0 - rb.hi[0]), 0.0);
          const double e1 = fmax(fmax(rb.lo[1] - q1, q1 - rb.hi[1]), 0.0);
          const double e2 = fmax(fmax(rb.lo[2] - q2, q2 - rb.hi[2]), 0.0);
          const bool need = live && !(e0 * e0 + e1 * e1 + e2 * e2 > best * kSlackLabel);
          if (!__any_sync(0xffffffffu, need)) continue;
#pragma unroll 4
          for (int32_t s = s0; s < s1; ++s) {
            const int64_t c = slot[s];
            const double ux = cen[3 * c] - q0, uy = cen[3 * c + 1] - q1, uz = cen[3 * c + 2] - q2;
            const double dd = ux * ux + uy * uy + uz * uz;
            if (dd < best || (dd == best && c < bi)) {
              best = dd;
              bi = c;
            }
          }
        }
      }
    }
    double bound = INFINITY;
    bool covered = true;
    face_bound(g, 0, c0, r, q0, bound, covered);
    face_bound(g, 1, c1, r, q1, bound, covered);
    face_bound(g, 2, c2, r, q2, bound, covered);
    const bool done = !live || covered || (bound > 0.0 && bound * bound > best * kSlackLabel);
    if (__all_sync(0xffffffffu, done)) break;
  }
  if (!live) return;
  const double vx = cen[3 * bi] - q0, vy = cen[3 * bi + 1] - q1, vz = cen[3 * bi + 2] - q2;
  const double dot = __dadd_rn(__dadd_rn(__dmul_rn(vx, nrm[3 * bi]), __dmul_rn(vy, nrm[3 * bi + 1])),
                               __dmul_rn(vz, nrm[3 * bi + 2]));
  out[((int64_t)ix * a.n[1] + iy) * a.n[2] + iz] = lab[2 * bi + (dot < 0.0 ? 1 : 0)] + 1.0;
}

// Bucket grid of about nc / 16 buckets over the query box (at most 2^21).
Buckets bucket_grid(const dm_box* b, int64_t nc) {
  Buckets g;
  double L[3], vol = 1.0;
  for (int d = 0; d < 3; ++d) {
    L[d] = b->hi[d] > b->lo[d] ? b->hi[d] - b->lo[d] : 1.0;
    vol *= L[d];
  }
  const double target = std::max<double>(1.0, std::min<double>((double)nc / 16.0, 1 << 21));
  const double h = cbrt(vol / target);
  for (int d = 0; d < 3; ++d) {
    g.n[d] = (int32_t)std::max(1.0, std::min(128.0, ceil(L[d] / h)));
    g.lo[d] = b->lo[d];
    g.inv[d] = g.n[d] / L[d];
    g.h[d] = L[d] / g.n[d];
  }
  return g;
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

namespace {
// Instance-mask workspace: status word, children (centroid, normal, labels: 8
// doubles), bucket counts / offsets / cursors and non-empty offsets (4 int32 per
// bucket), slots (1 int32 per child), bucket records.
size_t instance_layout(int64_t nc, int64_t nb, char* base, double** cen, int32_t** cnt,
                              int32_t** off, int32_t** cur, int32_t** nzo, int32_t** slot,
                              BucketRec** rec) {
  size_t o = 256;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o += (bytes + 255) / 256 * 256;
    return base ? base + at : nullptr;
  };
  char* c0 = take(sizeof(double) * 8 * (size_t)nc);
  char* c1 = take(sizeof(int32_t) * (size_t)(nb + 1));
  char* c2 = take(sizeof(int32_t) * (size_t)(nb + 1));
  char* c3 = take(sizeof(int32_t) * (size_t)(nb + 1));
  char* c4 = take(sizeof(int32_t) * (size_t)(nb + 1));
  char* c5 = take(sizeof(int32_t) * (size_t)nc);
  char* c6 = take(sizeof(BucketRec) * (size_t)nb);
  if (base) {
    *cen = (double*)c0;
    *cnt = (int32_t*)c1;
    *off = (int32_t*)c2;
    *cur = (int32_t*)c3;
    *nzo = (int32_t*)c4;
    *slot = (int32_t*)c5;
    *rec = (BucketRec*)c6;
  }
  return o;
}

}  // namespace

extern "C" {

size_t dm_mask_workspace_size(int64_t nt, int32_t levels, const dm_box* box) {
  if (nt < 0 || levels < 0 || levels > 8) return 0;
  if (!box) return 256;
  const int64_t nc = std::max<int64_t>(nt << (2 * levels), 1);
  const Buckets g = bucket_grid(box, nc);
  const int64_t nb = (int64_t)g.n[0] * g.n[1] * g.n[2];
  return instance_layout(nc, nb, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                         nullptr);
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
  if (ws_bytes < dm_mask_workspace_size(nt, levels, box)) return DM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t nc = nt << (2 * levels);
  if (nc >= (int64_t)INT32_MAX) return DM_ERR_SIZE;
  const Buckets g = bucket_grid(box, nc);
  const int64_t nb = (int64_t)g.n[0] * g.n[1] * g.n[2];
  char* w = (char*)workspace;
  int* err = (int*)w;
  double* cen;
  int32_t *cnt, *off, *cur, *nzo, *slot;
  BucketRec* rec;
  instance_layout(nc, nb, w, &cen, &cnt, &off, &cur, &nzo, &slot, &rec);
  double* nrm = cen + 3 * nc;
  double* lab = nrm + 3 * nc;
  k_children<<<(unsigned)cdiv(nc, kThreads), kThreads, 0, st>>>(verts, nv, faces, nt, levels,
                                                                 cen, nrm, lab, err);
  if (cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (size_t)(nb + 1), st) != cudaSuccess ||
      cudaMemsetAsync(cur, 0, sizeof(int32_t) * (size_t)(nb + 1), st) != cudaSuccess)
    return DM_ERR_CUDA;
  const unsigned gc = (unsigned)cdiv(nc, kThreads), gb = (unsigned)cdiv(nb, kThreads);
  k_bucket_count<<<gc, kThreads, 0, st>>>(cen, nc, g, cnt);
  k_scan<<<1, 1024, 0, st>>>(cnt, nb, 0, off);
  k_scan<<<1, 1024, 0, st>>>(cnt, nb, 1, nzo);  // nzo[nb] = non-empty buckets
  k_bucket_fill<<<gc, kThreads, 0, st>>>(cen, nc, g, off, cur, slot);
  k_bucket_boxes<<<gb, kThreads, 0, st>>>(off, nzo, slot, cen, nb, rec);
  const int64_t npts = (int64_t)box->shape[0] * box->shape[1] * box->shape[2];
  const int64_t bricks = cdiv(box->shape[0], kBrickX) * cdiv(box->shape[1], kBrickY) *
                         cdiv(box->shape[2], kBrickZ);
  k_nearest_label<<<(unsigned)cdiv(bricks * 32, kThreads), kThreads, 0, st>>>(
      cen, nrm, lab, slot, off, nzo, rec, g, make_axes(box), mask);
  count_launches(7);
  return status();
}

}  // extern "C"
