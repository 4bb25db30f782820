// meshFT forward without any device allocation by the library or the caller's
// workspace: the scratch lives in a fixed array compiled into this library.
//
// Who needs this: callers that are not allowed to allocate device memory at the
// time they render -- a host application whose memory manager owns every device
// byte (a fixed pool or a caching allocator that foreign code must not bypass),
// a service that allocates once at start-up and never again on its latency path,
// or a plugin boundary that can hand over only the input and output buffers.
// They still pass inputs and outputs; the intermediate face records and partial
// sums go to g_noalloc_scratch below.
//
// Limits and behaviour:
//  * the array is kNoAllocScratchBytes (8 MiB) on every GPU that loads this
//    library, held until the process exits; a request whose workspace would not
//    fit (dm_meshft_forward_workspace_size(nv, nt, n_band) > 8 MiB) is rejected
//    with DM_ERR_SIZE before anything is enqueued;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it; make that
//    first call before any stream capture;
//  * every call on a device shares the one array and it keeps the previous
//    call's contents: the status word at its start is cleared by each call, all
//    other scratch is fully rewritten before it is read; two calls whose work
//    overlaps on the GPU (different streams without ordering) race on it;
//  * faults the kernels detect (a face index out of range) set bits in that
//    status word; dm_meshft_forward_noalloc_device_error reads and clears it.
//    Every host-side argument check runs before anything is enqueued.
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "../../include/deltamic_b200.h"
#include "meshft_internal.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch per device (the host-side symbol is only a
// stand-in for it and must never be passed to a kernel).
std::atomic<void*> g_scratch_addr[kMaxDevices];

int scratch_for_current_device(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DM_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return DM_ERR_UNSUPPORTED;
  void* p = g_scratch_addr[dev].load();
  if (!p) {
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return DM_ERR_CUDA;
    g_scratch_addr[dev].store(p);
  }
  *out = p;
  return DM_OK;
}

}  // namespace

extern "C" int dm_meshft_forward_noalloc(const float* verts, int64_t nv, const int64_t* faces,
                                         int64_t nt, const float* faces_coeff,
                                         const dm_box* box, const int32_t* band_index,
                                         int64_t n_band, const float* otf, float* ft_list,
                                         float* grid, dm_stream_t stream) {
  const size_t need = dm_meshft_forward_workspace_size(nv, nt, n_band);
  if (need == 0) return DM_ERR_SIZE;              // sizes the kernels cannot index
  if (need > kNoAllocScratchBytes) return DM_ERR_SIZE;  // beyond the fixed scratch
  // the argument checks of dm_meshft_forward, repeated here so that a refused
  // call enqueues nothing (not even the status-word clear below)
  if (!dm::box_ok(box)) return DM_ERR_INVALID_ARG;
  if (nt > 0 && (!verts || !faces || !faces_coeff)) return DM_ERR_INVALID_ARG;
  if (n_band > 0 && (!band_index || !ft_list)) return DM_ERR_INVALID_ARG;
  void* scratch = nullptr;
  const int s = scratch_for_current_device(&scratch);
  if (s != DM_OK) return s;
  // the status word at the start of the scratch must start at zero each call
  if (cudaMemsetAsync(scratch, 0, 256, (cudaStream_t)stream) != cudaSuccess) return DM_ERR_CUDA;
  return dm_meshft_forward(verts, nv, faces, nt, faces_coeff, box, band_index, n_band, otf,
                           ft_list, grid, scratch, kNoAllocScratchBytes, stream);
}

extern "C" int dm_meshft_forward_noalloc_device_error(int* out_flags, dm_stream_t stream) {
  if (!out_flags) return DM_ERR_INVALID_ARG;
  void* scratch = nullptr;
  const int s = scratch_for_current_device(&scratch);
  if (s != DM_OK) return s;
  // the status word is the first int of the scratch (the forward's workspace layout)
  return dm_device_error(scratch, out_flags, stream);
}
