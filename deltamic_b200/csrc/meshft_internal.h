// Internal launch interface between the C ABI (capi.cu) and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "dm_common.cuh"

namespace dm {

// Tile-shape variants (picked per size class by the autotuner, dm_set_variants).
// Forward: R frequencies per thread, NT threads; face tiles of 64 in 3 stages.
// Backward: F faces per thread, NT threads; frequency tiles of 128 in 3 stages.
// ``waves``: items per launch as a multiple of the SM count.
struct FwdVariant {
  int R, NT, waves;
};
struct BwdVariant {
  int F, NT, waves;
  int minb = 0;  // CTAs per SM the register allocation must allow (0: no cap)
};
constexpr int kFwdTF = 64, kBwdTX = 128, kStages = 3;
constexpr int kNumFwdVariants = 6;
constexpr int kNumBwdVariants = 9;
constexpr FwdVariant kFwdVariants[kNumFwdVariants] = {
    {4, 128, 8}, {2, 128, 8}, {4, 256, 8}, {8, 64, 8}, {4, 128, 16}, {2, 256, 16}};
constexpr BwdVariant kBwdVariants[kNumBwdVariants] = {
    {2, 128, 8},    {1, 128, 8},    {2, 64, 8},     {1, 256, 8},   {2, 128, 16},
    {1, 128, 16},   {2, 128, 8, 5}, {2, 128, 16, 6}, {1, 128, 16, 8}};
int fwd_variant();
int bwd_variant();
void set_variants(int fwd, int bwd);

// Totals of a batched plan (sums over cells).
struct PlanTotals {
  int64_t nv, nt, nband, fpart, bpart, face_blks, band_blks, fwd_items, bwd_items;
  int32_t fwd_var = 0, bwd_var = 0;  // the tile variants the plan was made for
};

int num_sms();

// Host-side argument checks shared by the C-ABI entry points (capi.cu): a box
// with positive extents and shapes of at most INT32_MAX voxels and only known
// band flags; mesh and band sizes the kernels can index in int32.
bool box_ok(const dm_box* b);
bool sizes_ok(int64_t nv, int64_t nt, int64_t nband);

// Sequential carving of a caller's workspace into 256-byte aligned pieces (a
// null base only measures: take() returns null and advances the offset).
constexpr size_t kAlign = 256;
inline size_t up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }
struct Carve {
  char* base;
  size_t off;
  explicit Carve(void* p) : base((char*)p), off(0) {}
  template <typename T>
  T* take(size_t count) {
    T* p = base ? (T*)(base + off) : nullptr;
    off += up(sizeof(T) * (count > 0 ? count : 1));
    return p;
  }
};

// Topology (vertex <- face CSR) layout: status word, off[nv+1], ent[3nt],
// count[nv+1], cursor[nv+1]; returns its size in bytes.
struct TopoWs {
  int* err;
  int32_t* off;
  int32_t* ent;
  int32_t* count;
  int32_t* cursor;
};
size_t topo_layout(void* p, int64_t nv, int64_t nt, TopoWs* out);

// Instrumentation: launches counted per process; optional CUDA events around the
// main forward / backward kernels (kind 0 / 1).
void count_launches(int n);
void profile_begin(int kind, cudaStream_t st);
void profile_end(int kind, cudaStream_t st);
void set_band_half(CellDesc& d, bool herm);
void plan_cell_tiles(CellDesc& d);
void plan_cell_tiles_for(CellDesc& d, const FwdVariant& fv, const BwdVariant& bv);
void plan_offsets(CellDesc* cells, int ncells, PlanTotals& t);

int launch_face_prep(const Cells& c, const PlanTotals& t, const float* verts, const int64_t* faces,
                     const float* coeff, FaceRec* recs, double* area_part, int* err,
                     cudaStream_t st);
int launch_forward(const Cells& c, const PlanTotals& t, const FaceRec* recs,
                   const int32_t* band_index, const double* area_part, const float* otf,
                   float2* fpart, float2* ft_list, float2* grid, int* err, cudaStream_t st);
int launch_backward(const Cells& c, const PlanTotals& t, const float* verts, const int64_t* faces,
                    const float* coeff, const FaceRec* recs, const double* area_part,
                    const int32_t* band_index, const float2* grad_list, const float2* grad_grid,
                    const float* otf, float grad_scale, const float2* ft_list, XiRec* xrec,
                    double* s_part, float* bpart, float* contrib, const int32_t* csr_off,
                    const int32_t* csr_ent, float* grad_verts, float* grad_coeff,
                    float* grad_otf_band, int32_t* key_hist, int32_t* key_first,
                    int32_t* face_order, int32_t* face_slot, int* err, cudaStream_t st);
int launch_vertex_gather(int64_t nv, const int32_t* csr_off, const int32_t* csr_ent,
                         const float* contrib, float* grad_verts, cudaStream_t st);

// Surface + enclosed-volume transform (volume.cu): fixed tile shapes; plan_volume
// re-plans a single cell and sets t's part sizes and item counts for them.
void plan_volume(CellDesc& d, PlanTotals& t);
int launch_volume_forward(const CellDesc& d, const PlanTotals& t, const float* verts,
                          const int64_t* faces, const float* regint, const int32_t* band_index,
                          const float* otf, double* area_part, double* det_part, FaceRec* recs,
                          float4* vrec, float2* fpart, float2* ft_list, float2* vol_list,
                          float2* grid, int* err, cudaStream_t st);
int launch_volume_backward(const CellDesc& d, const PlanTotals& t, const float* verts,
                           const int64_t* faces, const float* regint, const int32_t* band_index,
                           const float2* grad_list, const float2* grad_grid, const float* otf,
                           float grad_scale, const float2* ft_list, const float2* vol_list,
                           double* area_part, double* det_part, double* s_part, FaceRec* recs,
                           float4* vrec, float4* fw, XiRec* xrec, float4* xg, float* bpart,
                           float* contrib, const int32_t* csr_off, const int32_t* csr_ent,
                           float* grad_verts, float* grad_regint, int* err, cudaStream_t st);
// Explicit float32 frequency lists (meshft.cu): one mesh, vertex coordinates as
// given, the cell (lower corner 0, lengths from the vertices) computed on the
// device into dev_desc; plan_xi_cell sizes the launches (t.nband = n_xi).
CellDesc plan_xi_cell(int64_t nv, int64_t nt, int64_t n_xi, PlanTotals& t);
int launch_xi_forward(const CellDesc& plan, const PlanTotals& t, const float* verts,
                      const int64_t* faces, const float* coeff, const float* xi_list,
                      CellDesc* dev_desc, FaceRec* recs, double* area_part, XiRecOff* xr,
                      float2* fpart, float2* ft_list, int* err, cudaStream_t st);
int launch_xi_backward(const CellDesc& plan, const PlanTotals& t, const float* verts,
                       const int64_t* faces, const float* coeff, const float* xi_list,
                       const float2* grad_list, float grad_scale, const float2* ft_list,
                       const int32_t* csr_off, const int32_t* csr_ent, CellDesc* dev_desc,
                       FaceRec* recs, double* area_part, XiRecOff* xr, double* s_part,
                       float* bpart, float* contrib, float* grad_verts, float* grad_coeff,
                       int32_t* key_hist, int32_t* key_first, int32_t* face_order,
                       int32_t* face_slot, int* err, cudaStream_t st);

// Float64 meshFT (meshft64.cu): one mesh, the frequencies of a grid band
// (band_index with the box) or of an explicit xi list (box NULL, vertices as
// given); every frequency evaluated.
struct Plan64 {
  CellDesc d;
  int64_t face_blks, band_blks, fpart, bpart, fwd_items, bwd_items;
};
Plan64 plan64(int64_t nv, int64_t nt, int64_t nfreq, const dm_box* box);
size_t face64_bytes();
size_t xi64_bytes();
int launch64_forward(const Plan64& p, const double* verts, const int64_t* faces,
                     const double* coeff, const int32_t* band_index, const double* xi_list,
                     const double* otf, void* recs, double* area_part, void* xrec, double* fpart,
                     double* ft_list, double* grid, int* err, cudaStream_t st);
int launch64_backward(const Plan64& p, const double* verts, const int64_t* faces,
                      const double* coeff, const int32_t* band_index, const double* xi_list,
                      const double* grad_list, const double* grad_grid, const double* otf,
                      double grad_scale, const double* ft_list, const int32_t* csr_off,
                      const int32_t* csr_ent, void* recs, double* area_part, void* xrec,
                      double* s_part, double* bpart, double* contrib, double* grad_verts,
                      double* grad_coeff, int* err, cudaStream_t st);

int launch_topology(const Cells& c, const PlanTotals& t, const int64_t* faces, int32_t* count,
                    int32_t* off, int32_t* cursor, int32_t* ent, int* err, cudaStream_t st);

}  // namespace dm
