// extern "C" entry points of libdeltamic_b200.so (declared in
// include/deltamic_b200.h): argument checks, workspace carving, launches.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <atomic>

#include "band_internal.h"
#include "dm_common.cuh"
#include "meshft_internal.h"

using namespace dm;

namespace dm {

bool box_ok(const dm_box* b) {
  if (!b) return false;
  if (b->band_flags & ~DM_BAND_HERMITIAN) return false;
  for (int d = 0; d < 3; ++d) {
    if (b->shape[d] <= 0) return false;
    if (!(b->hi[d] > b->lo[d])) return false;
  }
  const int64_t n = (int64_t)b->shape[0] * b->shape[1] * b->shape[2];
  return n <= (int64_t)INT32_MAX;
}

bool sizes_ok(int64_t nv, int64_t nt, int64_t nband) {
  return nv >= 0 && nt >= 0 && nband >= 0 && nv < (int64_t)INT32_MAX / 3 &&
         nt < (int64_t)INT32_MAX / 9 && nband < (int64_t)INT32_MAX;
}

size_t topo_layout(void* p, int64_t nv, int64_t nt, TopoWs* out) {
  Carve c(p);
  TopoWs w;
  w.err = c.take<int>(4);
  w.off = c.take<int32_t>(nv + 1);
  w.ent = c.take<int32_t>(3 * nt);
  w.count = c.take<int32_t>(nv + 1);
  w.cursor = c.take<int32_t>(nv + 1);
  if (out) *out = w;
  return c.off;
}

}  // namespace dm

namespace {

CellDesc single_cell(const dm_box* b, int64_t nv, int64_t nt, int64_t nband, PlanTotals& t) {
  CellDesc d;
  memset(&d, 0, sizeof(d));
  for (int k = 0; k < 3; ++k) {
    d.lo[k] = b ? b->lo[k] : 0.0;
    d.len[k] = b ? b->hi[k] - b->lo[k] : 1.0;
    d.n[k] = b ? b->shape[k] : 1;
  }
  d.nv = (int32_t)nv;
  d.nt = (int32_t)nt;
  d.nband = (int32_t)nband;
  set_band_half(d, b && (b->band_flags & DM_BAND_HERMITIAN));
  d.grid_off = 0;
  plan_offsets(&d, 1, t);
  return d;
}

// Totals of the larger of the full-band and half-band plans: the workspace
// queries see no box, so their sizes cover either.
void plan_any(int64_t nv, int64_t nt, int64_t nband, PlanTotals& t) {
  PlanTotals a, h;
  dm_box b;
  memset(&b, 0, sizeof(b));
  for (int k = 0; k < 3; ++k) {
    b.hi[k] = 1.0;
    b.shape[k] = 1;
  }
  single_cell(&b, nv, nt, nband, a);
  b.band_flags = DM_BAND_HERMITIAN;
  single_cell(&b, nv, nt, nband, h);
  t = a;
  t.fpart = std::max(a.fpart, h.fpart);
  t.bpart = std::max(a.bpart, h.bpart);
}

Cells one_cell(const CellDesc& d) {
  Cells c;
  c.p = nullptr;
  c.n = 1;
  c.one = d;
  return c;
}

// Forward workspace layout.
struct FwdWs {
  int* err;
  double* area_part;
  FaceRec* recs;
  float2* fpart;
};
size_t fwd_layout(void* ws, const PlanTotals& t, FwdWs* out) {
  Carve c(ws);
  FwdWs w;
  w.err = c.take<int>(4);
  w.area_part = c.take<double>(t.face_blks);
  w.recs = c.take<FaceRec>(t.nt);
  w.fpart = c.take<float2>(t.fpart);
  if (out) *out = w;
  return c.off;
}

struct BwdWs {
  int* err;
  double* area_part;
  double* s_part;
  FaceRec* recs;
  XiRec* xrec;
  float* bpart;
  float* contrib;
  int32_t* key_hist;    // [face_blks][256]
  int32_t* key_first;   // [face_blks][256]
  int32_t* face_order;  // [nt]
  int32_t* face_slot;   // [nt]
  void* topo;
};
size_t bwd_layout(void* ws, const PlanTotals& t, BwdWs* out) {
  Carve c(ws);
  BwdWs w;
  w.err = c.take<int>(4);
  w.area_part = c.take<double>(t.face_blks);
  w.s_part = c.take<double>(t.band_blks);
  w.recs = c.take<FaceRec>(t.nt);
  w.xrec = c.take<XiRec>(t.nband);
  w.bpart = c.take<float>(t.bpart);
  w.contrib = c.take<float>(9 * t.nt);
  w.key_hist = c.take<int32_t>(256 * t.face_blks);
  w.key_first = c.take<int32_t>(256 * t.face_blks);
  w.face_order = c.take<int32_t>(t.nt);
  w.face_slot = c.take<int32_t>(t.nt);
  w.topo = c.base ? (void*)(c.base + c.off) : nullptr;
  c.off += topo_layout(nullptr, t.nv, t.nt, nullptr);
  if (out) *out = w;
  return c.off;
}

}  // namespace

// ---------------------------------------------------------------------------
// Instrumentation state (process-wide, current device only).
namespace dm {
namespace {
std::atomic<long long> g_launches{0};
constexpr int kProfRing = 512;
struct ProfRing {
  cudaEvent_t ev[kProfRing][2];
  int n = 0;        // pairs recorded since the last read
  bool ready = false;
};
int g_profile_on = 0;
ProfRing g_prof[2];
int g_pending[2] = {-1, -1};
}  // namespace

void count_launches(int n) { g_launches += n; }

void profile_begin(int kind, cudaStream_t st) {
  if (!g_profile_on || kind < 0 || kind > 1) return;
  ProfRing& r = g_prof[kind];
  if (!r.ready) {
    for (int i = 0; i < kProfRing; ++i) {
      cudaEventCreate(&r.ev[i][0]);
      cudaEventCreate(&r.ev[i][1]);
    }
    r.ready = true;
  }
  if (r.n >= kProfRing) return;
  cudaEventRecord(r.ev[r.n][0], st);
  g_pending[kind] = r.n;
}

void profile_end(int kind, cudaStream_t st) {
  if (!g_profile_on || kind < 0 || kind > 1 || g_pending[kind] < 0) return;
  ProfRing& r = g_prof[kind];
  cudaEventRecord(r.ev[g_pending[kind]][1], st);
  r.n += 1;
  g_pending[kind] = -1;
}
}  // namespace dm

// Workspace plans of the surface + enclosed-volume transform (volume.cu).
namespace {

CellDesc volume_cell(const dm_box* b, int64_t nv, int64_t nt, int64_t nband, PlanTotals& t) {
  CellDesc d = single_cell(b, nv, nt, nband, t);
  plan_volume(d, t);
  return d;
}

// Part sizes of the larger of the full-band and half-band plans (no box).
void volume_plan_any(int64_t nv, int64_t nt, int64_t nband, PlanTotals& t) {
  dm_box b;
  memset(&b, 0, sizeof(b));
  for (int k = 0; k < 3; ++k) {
    b.hi[k] = 1.0;
    b.shape[k] = 1;
  }
  PlanTotals a, h;
  volume_cell(&b, nv, nt, nband, a);
  b.band_flags = DM_BAND_HERMITIAN;
  volume_cell(&b, nv, nt, nband, h);
  t = a;
  t.fpart = std::max(a.fpart, h.fpart);
  t.bpart = std::max(a.bpart, h.bpart);
}

struct VolFwdWs {
  int* err;
  double* area_part;
  double* det_part;
  FaceRec* recs;
  float4* vrec;
  float2* fpart;
};
size_t vol_fwd_layout(void* ws, const PlanTotals& t, VolFwdWs* out) {
  Carve c(ws);
  VolFwdWs w;
  w.err = c.take<int>(4);
  w.area_part = c.take<double>(t.face_blks);
  w.det_part = c.take<double>(t.face_blks);
  w.recs = c.take<FaceRec>(t.nt);
  w.vrec = c.take<float4>(t.nt);
  w.fpart = c.take<float2>(t.fpart);
  if (out) *out = w;
  return c.off;
}

struct VolBwdWs {
  int* err;
  double* area_part;
  double* det_part;
  double* s_part;  // [3][band_blks]
  FaceRec* recs;
  float4* vrec;
  float4* fw;
  XiRec* xrec;
  float4* xg;
  float* bpart;
  float* contrib;
  void* topo;
};
size_t vol_bwd_layout(void* ws, const PlanTotals& t, VolBwdWs* out) {
  Carve c(ws);
  VolBwdWs w;
  w.err = c.take<int>(4);
  w.area_part = c.take<double>(t.face_blks);
  w.det_part = c.take<double>(t.face_blks);
  w.s_part = c.take<double>(3 * t.band_blks);
  w.recs = c.take<FaceRec>(t.nt);
  w.vrec = c.take<float4>(t.nt);
  w.fw = c.take<float4>(t.nt);
  w.xrec = c.take<XiRec>(t.nband);
  w.xg = c.take<float4>(t.nband);
  w.bpart = c.take<float>(t.bpart);
  w.contrib = c.take<float>(9 * t.nt);
  w.topo = c.base ? (void*)(c.base + c.off) : nullptr;
  c.off += topo_layout(nullptr, t.nv, t.nt, nullptr);
  if (out) *out = w;
  return c.off;
}

}  // namespace

extern "C" {

int dm_profile_enable(int enable) {
  dm::g_profile_on = enable ? 1 : 0;
  for (int k = 0; k < 2; ++k) dm::g_prof[k].n = 0;
  return DM_OK;
}

int dm_profile_read(int kernel, int* count, float* total_ms) {
  if (kernel < 0 || kernel > 1 || !count || !total_ms) return DM_ERR_INVALID_ARG;
  dm::ProfRing& r = dm::g_prof[kernel];
  float tot = 0.f;
  for (int i = 0; i < r.n; ++i) {
    if (cudaEventSynchronize(r.ev[i][1]) != cudaSuccess) return DM_ERR_CUDA;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, r.ev[i][0], r.ev[i][1]) != cudaSuccess) return DM_ERR_CUDA;
    tot += ms;
  }
  *count = r.n;
  *total_ms = tot;
  r.n = 0;
  return DM_OK;
}

long long dm_launch_count(void) { return dm::g_launches.load(); }

int dm_set_variants(int fwd, int bwd) {
  if (fwd < 0 || fwd >= dm::kNumFwdVariants || bwd < 0 || bwd >= dm::kNumBwdVariants)
    return DM_ERR_INVALID_ARG;
  dm::set_variants(fwd, bwd);
  return DM_OK;
}

int dm_get_variants(int* fwd, int* bwd, int* n_fwd, int* n_bwd) {
  if (fwd) *fwd = dm::fwd_variant();
  if (bwd) *bwd = dm::bwd_variant();
  if (n_fwd) *n_fwd = dm::kNumFwdVariants;
  if (n_bwd) *n_bwd = dm::kNumBwdVariants;
  return DM_OK;
}


int dm_abi_version(void) { return 2; }

const char* dm_status_string(int status) {
  if (status == DM_OK) return "ok";
  if (status & DM_ERR_INVALID_ARG) return "invalid argument";
  if (status & DM_ERR_BAD_INDEX) return "face index out of range";
  if (status & DM_ERR_SIZE) return "size out of range";
  if (status & DM_ERR_WORKSPACE) return "workspace too small";
  if (status & DM_ERR_CUDA) return "CUDA error";
  if (status & DM_ERR_TIMEOUT) return "bounded device wait timed out";
  if (status & DM_ERR_UNSUPPORTED) return "unsupported";
  if (status & DM_ERR_NONFINITE) return "vertex coordinate not finite";
  return "unknown status";
}

int dm_device_error(void* workspace, int* out_flags, dm_stream_t stream) {
  if (!workspace || !out_flags) return DM_ERR_INVALID_ARG;
  int v = 0;
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemcpyAsync(&v, workspace, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return DM_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return DM_ERR_CUDA;
  if (cudaMemsetAsync(workspace, 0, sizeof(int), st) != cudaSuccess) return DM_ERR_CUDA;
  *out_flags = v;
  return DM_OK;
}

// ---------------------------------------------------------------------------
size_t dm_narrowband_workspace_size(int64_t n_voxels) {
  if (n_voxels < 0) return 0;
  const int64_t nb = band_blocks(n_voxels);
  return up(sizeof(int) * 4) + 2 * up(sizeof(int32_t) * std::max<int64_t>(nb, 1));
}

int dm_narrowband_compact(const float* otf, int64_t n_voxels, float thresh, int32_t* band_index,
                          int64_t* band_count, void* workspace, size_t ws_bytes,
                          dm_stream_t stream) {
  if (n_voxels < 0 || !band_count || !workspace || (n_voxels > 0 && (!otf || !band_index)))
    return DM_ERR_INVALID_ARG;
  if (n_voxels > (int64_t)INT32_MAX) return DM_ERR_SIZE;
  if (ws_bytes < dm_narrowband_workspace_size(n_voxels)) return DM_ERR_WORKSPACE;
  const int64_t nb = std::max<int64_t>(band_blocks(n_voxels), 1);
  Carve c(workspace);
  c.take<int>(4);
  int32_t* bc = c.take<int32_t>(nb);
  int32_t* bo = c.take<int32_t>(nb);
  return launch_narrowband(otf, n_voxels, thresh, band_index, band_count, bc, bo,
                           (cudaStream_t)stream);
}

int dm_narrowband_compact64(const double* otf, int64_t n_voxels, double thresh,
                            int32_t* band_index, int64_t* band_count, void* workspace,
                            size_t ws_bytes, dm_stream_t stream) {
  if (n_voxels < 0 || !band_count || !workspace || (n_voxels > 0 && (!otf || !band_index)))
    return DM_ERR_INVALID_ARG;
  if (n_voxels > (int64_t)INT32_MAX) return DM_ERR_SIZE;
  if (ws_bytes < dm_narrowband_workspace_size(n_voxels)) return DM_ERR_WORKSPACE;
  const int64_t nb = std::max<int64_t>(band_blocks(n_voxels), 1);
  Carve c(workspace);
  c.take<int>(4);
  int32_t* bc = c.take<int32_t>(nb);
  int32_t* bo = c.take<int32_t>(nb);
  return launch_narrowband64(otf, n_voxels, thresh, band_index, band_count, bc, bo,
                             (cudaStream_t)stream);
}

int dm_narrowband_hermitian(const int32_t* band_index, int64_t n_band, int64_t n_voxels,
                            int32_t* is_hermitian, dm_stream_t stream) {
  if (!is_hermitian || n_band < 0 || n_voxels < 0 || n_band > n_voxels ||
      (n_band > 0 && !band_index))
    return DM_ERR_INVALID_ARG;
  return launch_band_mirror(band_index, n_band, n_voxels, is_hermitian, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
size_t dm_topology_size(int64_t nv, int64_t nt) {
  if (nv < 0 || nt < 0) return 0;
  return topo_layout(nullptr, nv, nt, nullptr);
}

int dm_topology_build(const int64_t* faces, int64_t nt, int64_t nv, void* topology,
                      size_t topo_bytes, dm_stream_t stream) {
  if (!topology || (nt > 0 && !faces) || !sizes_ok(nv, nt, 0)) return DM_ERR_INVALID_ARG;
  if (topo_bytes < dm_topology_size(nv, nt)) return DM_ERR_WORKSPACE;
  PlanTotals t;
  CellDesc d = single_cell(nullptr, nv, nt, 0, t);
  TopoWs w;
  topo_layout(topology, nv, nt, &w);
  return launch_topology(one_cell(d), t, faces, w.count, w.off, w.cursor, w.ent, w.err,
                         (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
size_t dm_meshft_forward_workspace_size(int64_t nv, int64_t nt, int64_t n_band) {
  if (!sizes_ok(nv, nt, n_band)) return 0;
  PlanTotals t;
  plan_any(nv, nt, n_band, t);
  return fwd_layout(nullptr, t, nullptr);
}

int dm_meshft_forward(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                      const float* faces_coeff, const dm_box* box, const int32_t* band_index,
                      int64_t n_band, const float* otf, float* ft_list, float* grid,
                      void* workspace, size_t ws_bytes, dm_stream_t stream) {
  if (!sizes_ok(nv, nt, n_band)) return DM_ERR_SIZE;
  if (!box_ok(box) || !workspace) return DM_ERR_INVALID_ARG;
  if (nt > 0 && (!verts || !faces || !faces_coeff)) return DM_ERR_INVALID_ARG;
  if (n_band > 0 && (!band_index || !ft_list)) return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm_meshft_forward_workspace_size(nv, nt, n_band)) return DM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  PlanTotals t;
  CellDesc d = single_cell(box, nv, nt, n_band, t);
  FwdWs w;
  fwd_layout(workspace, t, &w);
  const Cells c = one_cell(d);
  int s = launch_face_prep(c, t, verts, faces, faces_coeff, w.recs, w.area_part, w.err, st);
  if (s) return s;
  return launch_forward(c, t, w.recs, band_index, w.area_part, otf, w.fpart, (float2*)ft_list,
                        (float2*)grid, w.err, st);
}

// ---------------------------------------------------------------------------
// Batches

static PlanTotals totals_of(const dm_batch* b) {
  PlanTotals t;
  t.nv = b->plan[0];
  t.nt = b->plan[1];
  t.nband = b->plan[2];
  t.fpart = b->plan[3];
  t.bpart = b->plan[4];
  t.face_blks = b->plan[5];
  t.band_blks = b->plan[6];
  t.fwd_items = b->plan[7];
  t.bwd_items = b->plan[8];
  t.fwd_var = (int32_t)b->plan[10];
  t.bwd_var = (int32_t)b->plan[11];
  return t;
}

static Cells cells_of(const dm_batch* b) {
  Cells c;
  memset(&c, 0, sizeof(c));
  c.p = (const CellDesc*)b->cells;
  c.n = b->ncells;
  return c;
}

static bool batch_ok(const dm_batch* b) { return b && b->ncells > 0 && b->cells; }

size_t dm_batch_desc_size(int ncells) {
  return ncells > 0 ? sizeof(CellDesc) * (size_t)ncells : 0;
}

int dm_batch_plan(const dm_cell* cells, int ncells, void* desc, size_t desc_bytes,
                  dm_batch* out, dm_stream_t stream) {
  if (!cells || ncells <= 0 || !desc || !out) return DM_ERR_INVALID_ARG;
  if (desc_bytes < dm_batch_desc_size(ncells)) return DM_ERR_WORKSPACE;
  CellDesc* d = new CellDesc[ncells];
  int64_t grid_end = 0, max_grid = 0;
  for (int i = 0; i < ncells; ++i) {
    const dm_cell& c = cells[i];
    if (!sizes_ok(c.nv, c.nt, c.n_band) || !box_ok(&c.box) || c.grid_offset < 0) {
      delete[] d;
      return DM_ERR_INVALID_ARG;
    }
    memset(&d[i], 0, sizeof(CellDesc));
    for (int k = 0; k < 3; ++k) {
      d[i].lo[k] = c.box.lo[k];
      d[i].len[k] = c.box.hi[k] - c.box.lo[k];
      d[i].n[k] = c.box.shape[k];
    }
    d[i].nv = (int32_t)c.nv;
    d[i].nt = (int32_t)c.nt;
    d[i].nband = (int32_t)c.n_band;
    set_band_half(d[i], (c.box.band_flags & DM_BAND_HERMITIAN) != 0);
    d[i].grid_off = c.grid_offset;
    const int64_t g = (int64_t)c.box.shape[0] * c.box.shape[1] * c.box.shape[2];
    grid_end = std::max(grid_end, c.grid_offset + g);
    max_grid = std::max(max_grid, g);
  }
  PlanTotals t;
  plan_offsets(d, ncells, t);
  if (t.nv >= (int64_t)INT32_MAX / 3 || t.nt >= (int64_t)INT32_MAX / 9 ||
      t.nband >= (int64_t)INT32_MAX || grid_end >= (int64_t)INT32_MAX ||
      t.fwd_items >= (int64_t)INT32_MAX || t.bwd_items >= (int64_t)INT32_MAX) {
    delete[] d;
    return DM_ERR_SIZE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const bool ok = cudaMemcpyAsync(desc, d, sizeof(CellDesc) * ncells, cudaMemcpyHostToDevice,
                                  st) == cudaSuccess &&
                  cudaStreamSynchronize(st) == cudaSuccess;
  delete[] d;
  if (!ok) return DM_ERR_CUDA;
  memset(out, 0, sizeof(*out));
  out->ncells = ncells;
  out->nv = t.nv;
  out->nt = t.nt;
  out->n_band = t.nband;
  out->grid_elems = grid_end;
  out->fwd_workspace = (int64_t)fwd_layout(nullptr, t, nullptr);
  out->bwd_workspace = (int64_t)bwd_layout(nullptr, t, nullptr);
  out->topology_bytes = (int64_t)topo_layout(nullptr, t.nv, t.nt, nullptr);
  out->image_workspace = (int64_t)image_ws_bytes_segs(max_grid, ncells);
  const int64_t p[9] = {t.nv, t.nt, t.nband, t.fpart, t.bpart,
                        t.face_blks, t.band_blks, t.fwd_items, t.bwd_items};
  for (int k = 0; k < 9; ++k) out->plan[k] = p[k];
  out->plan[9] = max_grid;
  out->plan[10] = t.fwd_var;  // launches use the variants the tiles were planned for
  out->plan[11] = t.bwd_var;
  out->cells = desc;
  return DM_OK;
}

int dm_batched_topology_build(const dm_batch* batch, const int64_t* faces, void* topology,
                              size_t topo_bytes, dm_stream_t stream) {
  if (!batch_ok(batch) || !topology || (batch->nt > 0 && !faces)) return DM_ERR_INVALID_ARG;
  if (topo_bytes < (size_t)batch->topology_bytes) return DM_ERR_WORKSPACE;
  const PlanTotals t = totals_of(batch);
  TopoWs w;
  topo_layout(topology, t.nv, t.nt, &w);
  return launch_topology(cells_of(batch), t, faces, w.count, w.off, w.cursor, w.ent, w.err,
                         (cudaStream_t)stream);
}

int dm_batched_meshft_forward(const dm_batch* batch, const float* verts, const int64_t* faces,
                              const float* faces_coeff, const int32_t* band_index,
                              const float* otf, float* ft_list, float* grid, void* workspace,
                              size_t ws_bytes, dm_stream_t stream) {
  if (!batch_ok(batch) || !workspace) return DM_ERR_INVALID_ARG;
  if (batch->nt > 0 && (!verts || !faces || !faces_coeff)) return DM_ERR_INVALID_ARG;
  if (batch->n_band > 0 && (!band_index || !ft_list)) return DM_ERR_INVALID_ARG;
  if (ws_bytes < (size_t)batch->fwd_workspace) return DM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const PlanTotals t = totals_of(batch);
  const Cells c = cells_of(batch);
  FwdWs w;
  fwd_layout(workspace, t, &w);
  int s = launch_face_prep(c, t, verts, faces, faces_coeff, w.recs, w.area_part, w.err, st);
  if (s) return s;
  return launch_forward(c, t, w.recs, band_index, w.area_part, otf, w.fpart, (float2*)ft_list,
                        (float2*)grid, w.err, st);
}

int dm_batched_meshft_backward(const dm_batch* batch, const float* verts, const int64_t* faces,
                               const float* faces_coeff, const int32_t* band_index,
                               const float* grad_list, const float* grad_grid, const float* otf,
                               float grad_scale, const float* ft_list, const void* topology,
                               float* grad_verts, float* grad_coeff, float* grad_otf_band,
                               void* workspace, size_t ws_bytes, dm_stream_t stream) {
  if (!batch_ok(batch) || !workspace || !topology) return DM_ERR_INVALID_ARG;
  if (batch->nt > 0 && (!verts || !faces || !faces_coeff)) return DM_ERR_INVALID_ARG;
  if (batch->nv > 0 && !grad_verts) return DM_ERR_INVALID_ARG;
  if (batch->n_band > 0 && (!band_index || !ft_list || (!grad_list && !grad_grid)))
    return DM_ERR_INVALID_ARG;
  if (ws_bytes < (size_t)batch->bwd_workspace) return DM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const PlanTotals t = totals_of(batch);
  const Cells c = cells_of(batch);
  BwdWs w;
  bwd_layout(workspace, t, &w);
  TopoWs tw;
  topo_layout(const_cast<void*>(topology), t.nv, t.nt, &tw);
  int s = launch_face_prep(c, t, verts, faces, faces_coeff, w.recs, w.area_part, w.err, st);
  if (s) return s;
  return launch_backward(c, t, verts, faces, faces_coeff, w.recs, w.area_part, band_index,
                         (const float2*)grad_list, (const float2*)grad_grid, otf, grad_scale,
                         (const float2*)ft_list, w.xrec, w.s_part, w.bpart, w.contrib, tw.off,
                         tw.ent, grad_verts, grad_coeff, grad_otf_band, w.key_hist,
                         w.key_first, w.face_order, w.face_slot, w.err, st);
}

int dm_batched_image_loss(const dm_batch* batch, const float* z, int kind, const float* target,
                          float contrast, float* image, float* loss, float* grad_z,
                          void* workspace, size_t ws_bytes, dm_stream_t stream) {
  if (!batch_ok(batch) || !z || !loss || !workspace) return DM_ERR_INVALID_ARG;
  if ((kind != 0 && kind != 1) || (kind == 1 && !target)) return DM_ERR_INVALID_ARG;
  if (ws_bytes < (size_t)batch->image_workspace) return DM_ERR_WORKSPACE;
  return launch_image_loss_cells((const CellDesc*)batch->cells, batch->ncells, batch->plan[9],
                                 (const float2*)z, kind, target, contrast, image, loss,
                                 (float2*)grad_z, workspace, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
size_t dm_meshft_backward_workspace_size(int64_t nv, int64_t nt, int64_t n_band) {
  if (!sizes_ok(nv, nt, n_band)) return 0;
  PlanTotals t;
  plan_any(nv, nt, n_band, t);
  return bwd_layout(nullptr, t, nullptr);
}

int dm_meshft_backward(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                       const float* faces_coeff, const dm_box* box, const int32_t* band_index,
                       int64_t n_band, const float* grad_list, const float* grad_grid,
                       const float* otf, float grad_scale, const float* ft_list,
                       const void* topology, float* grad_verts, float* grad_coeff,
                       float* grad_otf_band, void* workspace, size_t ws_bytes,
                       dm_stream_t stream) {
  if (!sizes_ok(nv, nt, n_band)) return DM_ERR_SIZE;
  if (!box_ok(box) || !workspace) return DM_ERR_INVALID_ARG;
  if (nt > 0 && (!verts || !faces || !faces_coeff)) return DM_ERR_INVALID_ARG;
  if (nv > 0 && !grad_verts) return DM_ERR_INVALID_ARG;
  if (n_band > 0 && (!band_index || !ft_list || (!grad_list && !grad_grid)))
    return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm_meshft_backward_workspace_size(nv, nt, n_band)) return DM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  PlanTotals t;
  CellDesc d = single_cell(box, nv, nt, n_band, t);
  BwdWs w;
  bwd_layout(workspace, t, &w);
  const Cells c = one_cell(d);
  const void* topo = topology;
  if (!topo) {
    TopoWs tw;
    topo_layout(w.topo, nv, nt, &tw);
    int s = launch_topology(c, t, faces, tw.count, tw.off, tw.cursor, tw.ent, w.err, st);
    if (s) return s;
    topo = w.topo;
  }
  TopoWs tw;
  topo_layout(const_cast<void*>(topo), nv, nt, &tw);
  int s = launch_face_prep(c, t, verts, faces, faces_coeff, w.recs, w.area_part, w.err, st);
  if (s) return s;
  return launch_backward(c, t, verts, faces, faces_coeff, w.recs, w.area_part, band_index,
                         (const float2*)grad_list, (const float2*)grad_grid, otf, grad_scale,
                         (const float2*)ft_list, w.xrec, w.s_part, w.bpart, w.contrib, tw.off,
                         tw.ent, grad_verts, grad_coeff, grad_otf_band, w.key_hist,
                         w.key_first, w.face_order, w.face_slot, w.err, st);
}

// ---------------------------------------------------------------------------
// Explicit float32 frequency lists.

namespace {

struct XiWs {
  int* err;
  CellDesc* desc;
  double* area_part;
  double* s_part;
  FaceRec* recs;
  XiRecOff* xr;
  float2* fpart;
  float* bpart;
  float* contrib;
  int32_t* key_hist;
  int32_t* key_first;
  int32_t* face_order;
  int32_t* face_slot;
  void* topo;
};

size_t xi_layout(void* ws, const PlanTotals& t, bool backward, XiWs* out) {
  Carve c(ws);
  XiWs w;
  memset(&w, 0, sizeof(w));
  w.err = c.take<int>(4);
  w.desc = c.take<CellDesc>(1);
  w.area_part = c.take<double>(t.face_blks);
  w.recs = c.take<FaceRec>(t.nt);
  w.xr = c.take<XiRecOff>(t.nband);
  if (!backward) {
    w.fpart = c.take<float2>(t.fpart);
  } else {
    w.s_part = c.take<double>(t.band_blks);
    w.bpart = c.take<float>(t.bpart);
    w.contrib = c.take<float>(9 * t.nt);
    w.key_hist = c.take<int32_t>(256 * t.face_blks);
    w.key_first = c.take<int32_t>(256 * t.face_blks);
    w.face_order = c.take<int32_t>(t.nt);
    w.face_slot = c.take<int32_t>(t.nt);
    w.topo = c.base ? (void*)(c.base + c.off) : nullptr;
    c.off += topo_layout(nullptr, t.nv, t.nt, nullptr);
  }
  if (out) *out = w;
  return c.off;
}

}  // namespace

size_t dm_meshft_forward_xi_workspace_size(int64_t nv, int64_t nt, int64_t n_xi) {
  if (!sizes_ok(nv, nt, n_xi)) return 0;
  PlanTotals t;
  plan_xi_cell(nv, nt, n_xi, t);
  return xi_layout(nullptr, t, false, nullptr);
}

int dm_meshft_forward_xi(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                         const float* faces_coeff, const float* xi_list, int64_t n_xi,
                         float* ft_list, void* workspace, size_t ws_bytes, dm_stream_t stream) {
  if (!sizes_ok(nv, nt, n_xi)) return DM_ERR_SIZE;
  if (!workspace) return DM_ERR_INVALID_ARG;
  if (nt > 0 && (!verts || !faces || !faces_coeff)) return DM_ERR_INVALID_ARG;
  if (n_xi > 0 && (!xi_list || !ft_list)) return DM_ERR_INVALID_ARG;
  if (nv > 0 && !verts) return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm_meshft_forward_xi_workspace_size(nv, nt, n_xi)) return DM_ERR_WORKSPACE;
  PlanTotals t;
  const CellDesc d = plan_xi_cell(nv, nt, n_xi, t);
  XiWs w;
  xi_layout(workspace, t, false, &w);
  return launch_xi_forward(d, t, verts, faces, faces_coeff, xi_list, w.desc, w.recs,
                           w.area_part, w.xr, w.fpart, (float2*)ft_list, w.err,
                           (cudaStream_t)stream);
}

size_t dm_meshft_backward_xi_workspace_size(int64_t nv, int64_t nt, int64_t n_xi) {
  if (!sizes_ok(nv, nt, n_xi)) return 0;
  PlanTotals t;
  plan_xi_cell(nv, nt, n_xi, t);
  return xi_layout(nullptr, t, true, nullptr);
}

int dm_meshft_backward_xi(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                          const float* faces_coeff, const float* grad_output_list,
                          const float* ftmesh_list, const float* xi_list, int64_t n_xi,
                          const void* topology, float* grad_verts, float* grad_coeff,
                          void* workspace, size_t ws_bytes, dm_stream_t stream) {
  if (!sizes_ok(nv, nt, n_xi)) return DM_ERR_SIZE;
  if (!workspace) return DM_ERR_INVALID_ARG;
  if (nt > 0 && (!verts || !faces || !faces_coeff)) return DM_ERR_INVALID_ARG;
  if (nv > 0 && (!grad_verts || !verts)) return DM_ERR_INVALID_ARG;
  if (n_xi > 0 && (!xi_list || !grad_output_list || !ftmesh_list)) return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm_meshft_backward_xi_workspace_size(nv, nt, n_xi)) return DM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  PlanTotals t;
  const CellDesc d = plan_xi_cell(nv, nt, n_xi, t);
  XiWs w;
  xi_layout(workspace, t, true, &w);
  const void* topo = topology;
  if (!topo && nt > 0) {
    PlanTotals tt;
    CellDesc dd = single_cell(nullptr, nv, nt, 0, tt);
    TopoWs tw;
    topo_layout(w.topo, nv, nt, &tw);
    const int s = launch_topology(one_cell(dd), tt, faces, tw.count, tw.off, tw.cursor, tw.ent,
                                  w.err, st);
    if (s) return s;
    topo = w.topo;
  }
  TopoWs tw;
  memset(&tw, 0, sizeof(tw));
  if (topo) topo_layout(const_cast<void*>(topo), nv, nt, &tw);
  if (grad_coeff && nt > 0 && n_xi == 0)
    cudaMemsetAsync(grad_coeff, 0, sizeof(float) * (size_t)nt, st);
  return launch_xi_backward(d, t, verts, faces, faces_coeff, xi_list,
                            (const float2*)grad_output_list, 1.0f, (const float2*)ftmesh_list,
                            tw.off, tw.ent, w.desc, w.recs, w.area_part, w.xr, w.s_part,
                            w.bpart, w.contrib, grad_verts, grad_coeff, w.key_hist,
                            w.key_first, w.face_order, w.face_slot, w.err, st);
}

// ---------------------------------------------------------------------------
// Float64 meshFT (meshft64.cu).

namespace {

struct Ws64 {
  int* err;
  double* area_part;
  void* recs;
  void* xrec;
  double* fpart;
  double* s_part;
  double* bpart;
  double* contrib;
  void* topo;
};

size_t ws64_layout(void* ws, const Plan64& p, bool backward, Ws64* out) {
  Carve c(ws);
  Ws64 w;
  memset(&w, 0, sizeof(w));
  w.err = c.take<int>(4);
  w.area_part = c.take<double>(p.face_blks);
  w.recs = c.take<char>(face64_bytes() * (size_t)std::max<int64_t>(p.d.nt, 1));
  w.xrec = c.take<char>(xi64_bytes() * (size_t)std::max<int64_t>(p.d.nband, 1));
  if (!backward) {
    w.fpart = c.take<double>(2 * (size_t)std::max<int64_t>(p.fpart, 1));
  } else {
    w.s_part = c.take<double>(p.band_blks);
    w.bpart = c.take<double>(p.bpart);
    w.contrib = c.take<double>(9 * (size_t)p.d.nt);
    w.topo = c.base ? (void*)(c.base + c.off) : nullptr;
    c.off += topo_layout(nullptr, p.d.nv, p.d.nt, nullptr);
  }
  if (out) *out = w;
  return c.off;
}

// Exactly one frequency source: grid band (box + band_index) or list (xi_list,
// no box); none needed without frequencies.
bool source64_ok(const dm_box* box, const int32_t* band_index, const double* xi_list,
                 int64_t n_freq) {
  if (band_index && xi_list) return false;
  if (band_index) return box_ok(box);
  if (xi_list) return box == nullptr;
  return n_freq == 0 && (box == nullptr || box_ok(box));
}

}  // namespace

size_t dm_meshft64_forward_workspace_size(int64_t nv, int64_t nt, int64_t n_freq) {
  if (!sizes_ok(nv, nt, n_freq)) return 0;
  return ws64_layout(nullptr, plan64(nv, nt, n_freq, nullptr), false, nullptr);
}

int dm_meshft64_forward(const double* verts, int64_t nv, const int64_t* faces, int64_t nt,
                        const double* faces_coeff, const dm_box* box, const int32_t* band_index,
                        const double* xi_list, int64_t n_freq, const double* otf,
                        double* ft_list, double* grid, void* workspace, size_t ws_bytes,
                        dm_stream_t stream) {
  if (!sizes_ok(nv, nt, n_freq)) return DM_ERR_SIZE;
  if (!workspace || !source64_ok(box, band_index, xi_list, n_freq)) return DM_ERR_INVALID_ARG;
  if (nt > 0 && (!verts || !faces || !faces_coeff)) return DM_ERR_INVALID_ARG;
  if (n_freq > 0 && !ft_list) return DM_ERR_INVALID_ARG;
  if (grid && !band_index) return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm_meshft64_forward_workspace_size(nv, nt, n_freq)) return DM_ERR_WORKSPACE;
  const Plan64 p = plan64(nv, nt, n_freq, band_index ? box : nullptr);
  Ws64 w;
  ws64_layout(workspace, p, false, &w);
  return launch64_forward(p, verts, faces, faces_coeff, band_index, xi_list, otf, w.recs,
                          w.area_part, w.xrec, w.fpart, ft_list, grid, w.err,
                          (cudaStream_t)stream);
}

size_t dm_meshft64_backward_workspace_size(int64_t nv, int64_t nt, int64_t n_freq) {
  if (!sizes_ok(nv, nt, n_freq)) return 0;
  return ws64_layout(nullptr, plan64(nv, nt, n_freq, nullptr), true, nullptr);
}

int dm_meshft64_backward(const double* verts, int64_t nv, const int64_t* faces, int64_t nt,
                         const double* faces_coeff, const dm_box* box,
                         const int32_t* band_index, const double* xi_list, int64_t n_freq,
                         const double* grad_list, const double* grad_grid, const double* otf,
                         double grad_scale, const double* ft_list, const void* topology,
                         double* grad_verts, double* grad_coeff, void* workspace,
                         size_t ws_bytes, dm_stream_t stream) {
  if (!sizes_ok(nv, nt, n_freq)) return DM_ERR_SIZE;
  if (!workspace || !source64_ok(box, band_index, xi_list, n_freq)) return DM_ERR_INVALID_ARG;
  if (nt > 0 && (!verts || !faces || !faces_coeff)) return DM_ERR_INVALID_ARG;
  if (nv > 0 && !grad_verts) return DM_ERR_INVALID_ARG;
  if (n_freq > 0 && (!ft_list || (!grad_list && !grad_grid))) return DM_ERR_INVALID_ARG;
  if (grad_grid && !band_index) return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm_meshft64_backward_workspace_size(nv, nt, n_freq)) return DM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const Plan64 p = plan64(nv, nt, n_freq, band_index ? box : nullptr);
  Ws64 w;
  ws64_layout(workspace, p, true, &w);
  const void* topo = topology;
  if (!topo && nt > 0) {
    PlanTotals t;
    CellDesc d = single_cell(nullptr, nv, nt, 0, t);
    TopoWs tw;
    topo_layout(w.topo, nv, nt, &tw);
    const int s = launch_topology(one_cell(d), t, faces, tw.count, tw.off, tw.cursor, tw.ent,
                                  w.err, st);
    if (s) return s;
    topo = w.topo;
  }
  TopoWs tw;
  memset(&tw, 0, sizeof(tw));
  if (topo) topo_layout(const_cast<void*>(topo), nv, nt, &tw);
  return launch64_backward(p, verts, faces, faces_coeff, band_index, xi_list, grad_list,
                           grad_grid, otf, grad_scale, ft_list, tw.off, tw.ent, w.recs,
                           w.area_part, w.xrec, w.s_part, w.bpart, w.contrib, grad_verts,
                           grad_coeff, w.err, st);
}

// ---------------------------------------------------------------------------
// Surface + enclosed-volume transform (volume.cu).

size_t dm_meshft_volume_forward_workspace_size(int64_t nv, int64_t nt, int64_t n_band) {
  if (!sizes_ok(nv, nt, n_band)) return 0;
  PlanTotals t;
  volume_plan_any(nv, nt, n_band, t);
  return vol_fwd_layout(nullptr, t, nullptr);
}

int dm_meshft_volume_forward(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                             const float* regint, const dm_box* box, const int32_t* band_index,
                             int64_t n_band, const float* otf, float* ft_list, float* vol_list,
                             float* grid, void* workspace, size_t ws_bytes,
                             dm_stream_t stream) {
  if (!sizes_ok(nv, nt, n_band)) return DM_ERR_SIZE;
  if (!box_ok(box) || !workspace || !regint) return DM_ERR_INVALID_ARG;
  if (nt > 0 && (!verts || !faces)) return DM_ERR_INVALID_ARG;
  if (n_band > 0 && (!band_index || !ft_list || !vol_list)) return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm_meshft_volume_forward_workspace_size(nv, nt, n_band)) return DM_ERR_WORKSPACE;
  PlanTotals t;
  const CellDesc d = volume_cell(box, nv, nt, n_band, t);
  VolFwdWs w;
  vol_fwd_layout(workspace, t, &w);
  return launch_volume_forward(d, t, verts, faces, regint, band_index, otf, w.area_part,
                               w.det_part, w.recs, w.vrec, w.fpart, (float2*)ft_list,
                               (float2*)vol_list, (float2*)grid, w.err, (cudaStream_t)stream);
}

size_t dm_meshft_volume_backward_workspace_size(int64_t nv, int64_t nt, int64_t n_band) {
  if (!sizes_ok(nv, nt, n_band)) return 0;
  PlanTotals t;
  volume_plan_any(nv, nt, n_band, t);
  return vol_bwd_layout(nullptr, t, nullptr);
}

int dm_meshft_volume_backward(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                              const float* regint, const dm_box* box, const int32_t* band_index,
                              int64_t n_band, const float* grad_list, const float* grad_grid,
                              const float* otf, float grad_scale, const float* ft_list,
                              const float* vol_list, const void* topology, float* grad_verts,
                              float* grad_regint, void* workspace, size_t ws_bytes,
                              dm_stream_t stream) {
  if (!sizes_ok(nv, nt, n_band)) return DM_ERR_SIZE;
  if (!box_ok(box) || !workspace || !regint) return DM_ERR_INVALID_ARG;
  if (nt > 0 && (!verts || !faces)) return DM_ERR_INVALID_ARG;
  if (nv > 0 && !grad_verts) return DM_ERR_INVALID_ARG;
  if (n_band > 0 && (!band_index || !ft_list || !vol_list || (!grad_list && !grad_grid)))
    return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm_meshft_volume_backward_workspace_size(nv, nt, n_band))
    return DM_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  PlanTotals t;
  const CellDesc d = volume_cell(box, nv, nt, n_band, t);
  VolBwdWs w;
  vol_bwd_layout(workspace, t, &w);
  const void* topo = topology;
  if (!topo) {
    TopoWs tw;
    topo_layout(w.topo, nv, nt, &tw);
    int s = launch_topology(one_cell(d), t, faces, tw.count, tw.off, tw.cursor, tw.ent, w.err,
                            st);
    if (s) return s;
    topo = w.topo;
  }
  TopoWs tw;
  topo_layout(const_cast<void*>(topo), nv, nt, &tw);
  return launch_volume_backward(d, t, verts, faces, regint, band_index,
                                (const float2*)grad_list, (const float2*)grad_grid, otf,
                                grad_scale, (const float2*)ft_list, (const float2*)vol_list,
                                w.area_part, w.det_part, w.s_part, w.recs, w.vrec, w.fw, w.xrec,
                                w.xg, w.bpart, w.contrib, tw.off, tw.ent, grad_verts,
                                grad_regint, w.err, st);
}

// ---------------------------------------------------------------------------
static bool axes_ok(const float* x0, int32_t n0, const float* x1, int32_t n1, const float* x2,
                    int32_t n2) {
  return x0 && x1 && x2 && n0 > 0 && n1 > 0 && n2 > 0 &&
         (int64_t)n0 * n1 * n2 <= (int64_t)INT32_MAX;
}

static bool axes_ok64(const double* x0, int32_t n0, const double* x1, int32_t n1,
                      const double* x2, int32_t n2) {
  return axes_ok((const float*)x0, n0, (const float*)x1, n1, (const float*)x2, n2);
}

int dm_gaussian_otf(const float* sigma, const float* xi0, int32_t n0, const float* xi1,
                    int32_t n1, const float* xi2, int32_t n2, float* otf, dm_stream_t stream) {
  if (!sigma || !otf || !axes_ok(xi0, n0, xi1, n1, xi2, n2)) return DM_ERR_INVALID_ARG;
  const float* xi[3] = {xi0, xi1, xi2};
  const int32_t n[3] = {n0, n1, n2};
  return launch_gaussian_otf(sigma, xi, n, otf, (cudaStream_t)stream);
}

size_t dm_gaussian_otf_grad_workspace_size(int64_t n) {
  if (n < 0) return 0;
  return up(sizeof(int) * 4) + up(sizeof(double) * 6 * (size_t)otf_grad_blocks(n));
}

int dm_gaussian_otf_sigma_grad(const float* grad_otf, const int32_t* band_index, int64_t n_band,
                               const float* otf, const float* xi0, int32_t n0, const float* xi1,
                               int32_t n1, const float* xi2, int32_t n2, float* grad_sigma,
                               void* workspace, size_t ws_bytes, dm_stream_t stream) {
  if (!otf || !grad_sigma || !workspace || !axes_ok(xi0, n0, xi1, n1, xi2, n2))
    return DM_ERR_INVALID_ARG;
  const int64_t nvox = (int64_t)n0 * n1 * n2;
  const int64_t n = band_index ? n_band : nvox;
  if (n < 0 || (n > 0 && !grad_otf)) return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm_gaussian_otf_grad_workspace_size(n)) return DM_ERR_WORKSPACE;
  Carve c(workspace);
  c.take<int>(4);
  double* part = c.take<double>(6 * (size_t)otf_grad_blocks(n));
  const float* xi[3] = {xi0, xi1, xi2};
  const int32_t nax[3] = {n0, n1, n2};
  return launch_otf_sigma_grad(grad_otf, band_index, n, otf, xi, nax, grad_sigma, part,
                               (cudaStream_t)stream);
}

int dm_gaussian_otf64(const double* sigma, const double* xi0, int32_t n0, const double* xi1,
                      int32_t n1, const double* xi2, int32_t n2, double* otf,
                      dm_stream_t stream) {
  if (!sigma || !otf || !axes_ok64(xi0, n0, xi1, n1, xi2, n2)) return DM_ERR_INVALID_ARG;
  const double* xi[3] = {xi0, xi1, xi2};
  const int32_t n[3] = {n0, n1, n2};
  return launch_gaussian_otf64(sigma, xi, n, otf, (cudaStream_t)stream);
}

int dm_gaussian_otf64_sigma_grad(const double* grad_otf, const int32_t* band_index,
                                 int64_t n_band, const double* otf, const double* xi0, int32_t n0,
                                 const double* xi1, int32_t n1, const double* xi2, int32_t n2,
                                 double* grad_sigma, void* workspace, size_t ws_bytes,
                                 dm_stream_t stream) {
  if (!otf || !grad_sigma || !workspace || !axes_ok64(xi0, n0, xi1, n1, xi2, n2))
    return DM_ERR_INVALID_ARG;
  const int64_t nvox = (int64_t)n0 * n1 * n2;
  const int64_t n = band_index ? n_band : nvox;
  if (n < 0 || (n > 0 && !grad_otf)) return DM_ERR_INVALID_ARG;
  if (ws_bytes < dm_gaussian_otf_grad_workspace_size(n)) return DM_ERR_WORKSPACE;
  Carve c(workspace);
  c.take<int>(4);
  double* part = c.take<double>(6 * (size_t)otf_grad_blocks(n));
  const double* xi[3] = {xi0, xi1, xi2};
  const int32_t nax[3] = {n0, n1, n2};
  return launch_otf_sigma_grad64(grad_otf, band_index, n, otf, xi, nax, grad_sigma, part,
                                 (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
size_t dm_image_loss_workspace_size(int64_t n) {
  if (n < 0) return 0;
  return image_ws_bytes(n);
}

int dm_image_loss(const float* z, int64_t n, int kind, const float* target, float contrast,
                  float* image, float* loss, float* grad_z, void* workspace, size_t ws_bytes,
                  dm_stream_t stream) {
  if (!z || n <= 0 || !loss || !workspace) return DM_ERR_INVALID_ARG;
  if (kind != 0 && kind != 1) return DM_ERR_INVALID_ARG;
  if (kind == 1 && !target) return DM_ERR_INVALID_ARG;
  if (n > (int64_t)INT32_MAX) return DM_ERR_SIZE;
  if (ws_bytes < dm_image_loss_workspace_size(n)) return DM_ERR_WORKSPACE;
  return launch_image_loss((const float2*)z, n, kind, target, contrast, image, loss,
                           (float2*)grad_z, workspace, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
int dm_voxelize(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                const dm_box* box, uint8_t* occupancy, int* status, dm_stream_t stream) {
  if (!box_ok(box) || !occupancy || nv < 0 || nt < 0 || (nt > 0 && (!verts || !faces)))
    return DM_ERR_INVALID_ARG;
  return launch_voxelize(verts, nv, faces, nt, *box, occupancy, status, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
int dm_adam_step(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, int64_t n,
                 float lr, float beta1, float beta2, float eps, int64_t* step,
                 dm_stream_t stream) {
  if (n < 0 || !step || (n > 0 && (!param || !grad || !exp_avg || !exp_avg_sq)))
    return DM_ERR_INVALID_ARG;
  return launch_adam(param, grad, exp_avg, exp_avg_sq, n, lr, beta1, beta2, eps, step,
                     (cudaStream_t)stream);
}

}  // extern "C"
