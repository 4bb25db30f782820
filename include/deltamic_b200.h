/*
 * deltamic_b200 -- C ABI of the B200 (sm_100a) mesh Fourier transform,
 * narrow-band, OTF and image-loss kernels.
 *
 * Conventions for every entry point:
 *  - all array arguments are DEVICE pointers (caller-owned, borrowed for the
 *    duration of the stream work), row-major and contiguous;
 *  - complex arrays are interleaved float pairs (re, im), i.e. complex64;
 *  - work is enqueued on ``stream`` and nothing synchronises, except the calls
 *    documented as synchronous (dm_device_error);
 *  - scratch memory is passed in as ``workspace`` / ``ws_bytes``; sizes come
 *    from the matching *_workspace_size query; nothing allocates device memory;
 *  - the return value is a status: 0 (DM_OK) or an OR of DM_ERR_* bits.  Host
 *    side argument checks return before anything is enqueued.  Faults detected
 *    on the device (out-of-range face indices, a bounded wait that ran out) set
 *    bits in a status word inside the workspace, read with dm_device_error.
 *
 * Frequencies are the centred grid of Fourier3dMesh (deltamic/render.py:153-172):
 *   xi_d[k] = (2k - (n_d - 1)) * pi / (box.hi[d] - box.lo[d]),  k = 0..n_d-1,
 * and a narrow band is a list of flat C-order voxel indices into that grid.
 */
#ifndef DELTAMIC_B200_H_
#define DELTAMIC_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* dm_stream_t; /* == cudaStream_t */

#define DM_OK 0
#define DM_ERR_INVALID_ARG 1   /* null pointer, negative size, bad dtype ... */
#define DM_ERR_BAD_INDEX 2     /* a face or band index out of range, or a broken band mirror */
#define DM_ERR_SIZE 4          /* a size beyond what the kernels index (int32 voxels) */
#define DM_ERR_WORKSPACE 8     /* workspace smaller than the query returned */
#define DM_ERR_CUDA 16         /* a CUDA launch or copy failed */
#define DM_ERR_TIMEOUT 32      /* a bounded device wait gave up */
#define DM_ERR_UNSUPPORTED 64  /* valid request this build does not serve */
#define DM_ERR_NONFINITE 128   /* a vertex coordinate is NaN or infinite (device status word) */

/* Box of a meshFT grid: box_size (render.py:116-123) and box_shape, plus the
 * properties of the narrow band passed with it. */
typedef struct dm_box {
  double lo[3];       /* box_size[:,0] */
  double hi[3];       /* box_size[:,1] */
  int32_t shape[3];   /* box_shape */
  int32_t band_flags; /* DM_BAND_* bits of the band passed with this box */
} dm_box;

/* The band is closed under xi -> -xi: with N voxels and the band in ascending
 * order, band_index[n_band-1-m] == N-1-band_index[m] for every m (the voxel of
 * -xi on the centred grid is N-1-idx).  Every OTF with OTF(-xi) == OTF(xi), the
 * Gaussian OTFs among them, gives such a band (dm_narrowband_hermitian tests
 * it).  The meshFT calls then evaluate the first (n_band+1)/2 frequencies only
 * and take the others from ft(-xi) = conj(ft(xi)) (the transform of a real
 * indicator); the backward folds the cotangent of -xi into xi the same way.
 * The kernels check the mirror relation and raise DM_ERR_BAD_INDEX where it
 * fails.  Without the bit every frequency is evaluated. */
#define DM_BAND_HERMITIAN 1

/* ABI version of this header (bumped on any signature change). */
int dm_abi_version(void);

/* Human-readable name of the lowest set error bit of ``status``. */
const char* dm_status_string(int status);

/* Synchronous: waits for ``stream``, then returns the device status word held in
 * a workspace of any of the calls below (and clears it).  *out_flags receives
 * the DM_ERR_* bits raised on the device. */
int dm_device_error(void* workspace, int* out_flags, dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * Narrow band.  Replaces the selection in MeshFTCUDA.forward
 * (deltamic/cuda_class.py:21-24): bool_filter = Filter > thresh, then the
 * frequency list gathered in C order.
 * band_index[0..count) receives the flat indices of voxels with otf > thresh in
 * ascending order (capacity n_voxels); *band_count (DEVICE int64) the count. */
size_t dm_narrowband_workspace_size(int64_t n_voxels);
int dm_narrowband_compact(const float* otf, int64_t n_voxels, float thresh,
                          int32_t* band_index, int64_t* band_count, void* workspace,
                          size_t ws_bytes, dm_stream_t stream);

/* The same selection on a float64 OTF (Fourier3dMesh(dtype=torch.float64)): the
 * comparison otf > thresh in double; workspace from dm_narrowband_workspace_size. */
int dm_narrowband_compact64(const double* otf, int64_t n_voxels, double thresh,
                            int32_t* band_index, int64_t* band_count, void* workspace,
                            size_t ws_bytes, dm_stream_t stream);

/* Asynchronous: *is_hermitian (DEVICE int32) = 1 if band_index[0..n_band) (of a
 * grid of n_voxels) is closed under xi -> -xi in the sense of DM_BAND_HERMITIAN,
 * else 0.  No counterpart in the reference, which evaluates every frequency. */
int dm_narrowband_hermitian(const int32_t* band_index, int64_t n_band, int64_t n_voxels,
                            int32_t* is_hermitian, dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * Vertex <- face incidence (CSR), built once per topology.  Replaces the host
 * loop that fills triangles_belonging_to_vertex_map / index_of_vertex_in_triangles
 * (deltamic/cpp/fourier3d_cuda_kernel.cu:487-501) without its 30-faces-per-vertex
 * cap.  Entries of a vertex are sorted by (face, corner), so the backward's
 * per-vertex sums run in a fixed order. */
size_t dm_topology_size(int64_t nv, int64_t nt);
int dm_topology_build(const int64_t* faces, int64_t nt, int64_t nv, void* topology,
                      size_t topo_bytes, dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * meshFT forward.  Replaces forward_fourier3d_cpp
 * (deltamic/cpp/fourier3d_cuda.cpp:27-42, :112-113; kernel .cu:281-311, host
 * prep .cu:42-51, :421-462) for frequencies on the grid of ``box``.
 *   verts[nv,3] float32 (unshifted: the box.lo shift of Fourier3dMesh.forward,
 *   render.py:144/148, is applied inside), faces[nt,3] int64, faces_coeff[nt],
 *   band_index[n_band] from dm_narrowband_compact.
 * Writes ft_list[n_band] (complex64).  If ``grid`` is not NULL it also writes
 * grid[band_index[m]] = ft_list[m] * (otf ? otf[band_index[m]] : 1); other grid
 * elements are left untouched (the caller zeroes the grid once). */
size_t dm_meshft_forward_workspace_size(int64_t nv, int64_t nt, int64_t n_band);
int dm_meshft_forward(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                      const float* faces_coeff, const dm_box* box, const int32_t* band_index,
                      int64_t n_band, const float* otf, float* ft_list, float* grid,
                      void* workspace, size_t ws_bytes, dm_stream_t stream);

/* meshFT forward for callers that cannot allocate device memory (no counterpart
 * in the reference).  Same arguments and results as dm_meshft_forward minus the
 * workspace: scratch is a fixed 8 MiB array inside this library (held on every
 * GPU that loads it).  Requests needing more workspace than that return
 * DM_ERR_SIZE before anything is enqueued.  The first call on a device looks up
 * the array's address (make it before any stream capture); calls share the
 * array, so calls that overlap on the GPU race. */
int dm_meshft_forward_noalloc(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                              const float* faces_coeff, const dm_box* box,
                              const int32_t* band_index, int64_t n_band, const float* otf,
                              float* ft_list, float* grid, dm_stream_t stream);

/* Synchronous: the device status word of dm_meshft_forward_noalloc on the current
 * device (DM_ERR_* bits set by its kernels, e.g. DM_ERR_BAD_INDEX for a face
 * index out of range), then cleared; the counterpart of dm_device_error for the
 * library's fixed scratch, whose address callers never see.  Each
 * dm_meshft_forward_noalloc call clears the word before its kernels run, so read
 * it after the call whose faults are wanted and before the next one. */
int dm_meshft_forward_noalloc_device_error(int* out_flags, dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * meshFT backward.  Replaces backward_fourier3d_cpp
 * (deltamic/cpp/fourier3d_cuda.cpp:44-65, :114; kernels .cu:314-416, host prep
 * .cu:16-36, :466-539) and adds the Faces_coeff and OTF gradients the reference
 * gets only from CPU autograd.
 * The cotangent on the band (PyTorch convention, dL/dRe + i dL/dIm) is
 *   g[m] = grad_scale * G[m] * (otf ? otf[band_index[m]] : 1),
 * with G[m] = grad_list[m] if grad_list != NULL, else grad_grid[band_index[m]].
 * ft_list is the forward's output.  topology from dm_topology_build (NULL: built
 * in the workspace on every call).
 * Writes grad_verts[nv,3]; optionally grad_coeff[nt] and
 * grad_otf_band[m] = grad_scale * Re(conj(G[m]) ft_list[m]). */
size_t dm_meshft_backward_workspace_size(int64_t nv, int64_t nt, int64_t n_band);
int dm_meshft_backward(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                       const float* faces_coeff, const dm_box* box, const int32_t* band_index,
                       int64_t n_band, const float* grad_list, const float* grad_grid,
                       const float* otf, float grad_scale, const float* ft_list,
                       const void* topology, float* grad_verts, float* grad_coeff,
                       float* grad_otf_band, void* workspace, size_t ws_bytes,
                       dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * meshFT on an explicit frequency list, float32: the reference FFI itself,
 * forward_fourier3d_cpp(Verts, Faces, Faces_coeff, xi_list) and
 * backward_fourier3d_cpp(Verts, Faces, Faces_coeff, grad_output_list,
 * ftmesh_list, xi_list) for scalar_t = float (deltamic/cpp/fourier3d_cuda.cpp:
 * 27-65, :112-115; kernels .cu:281-416).
 *   verts[nv,3] as given (no box shift: the caller passes Verts - box_size[:,0]
 *   as MeshFTCUDA does), faces[nt,3] int64, faces_coeff[nt], xi_list[n_xi,3] float32
 *   (any frequencies, on a grid or not).
 * forward writes ftmesh_list[n_xi] (complex64) = (2/M) sum_k A_k c_k F_k(xi).
 * backward takes grad_output_list[n_xi] (complex64, PyTorch convention) and the
 * forward's ftmesh_list, and writes grad_verts[nv,3] and, if not NULL,
 * grad_coeff[nt] (the reference returns only the vertex gradient).  topology
 * from dm_topology_build or NULL (built in the workspace).
 * Phases: the cell has lower corner 0 and length 2.5 max|v_d| per axis (found on
 * the device); each xi_d becomes m_d = xi_d L_d / pi, whose nearest integer
 * enters the exact 32-bit fixed-point phase and whose remainder a float term
 * below 3/8 of a turn (split phase).  A frequency with |m_d| >= 2^30 sets
 * DM_ERR_SIZE and a non-finite vertex DM_ERR_NONFINITE in the status word. */
size_t dm_meshft_forward_xi_workspace_size(int64_t nv, int64_t nt, int64_t n_xi);
int dm_meshft_forward_xi(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                         const float* faces_coeff, const float* xi_list, int64_t n_xi,
                         float* ftmesh_list, void* workspace, size_t ws_bytes,
                         dm_stream_t stream);
size_t dm_meshft_backward_xi_workspace_size(int64_t nv, int64_t nt, int64_t n_xi);
int dm_meshft_backward_xi(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                          const float* faces_coeff, const float* grad_output_list,
                          const float* ftmesh_list, const float* xi_list, int64_t n_xi,
                          const void* topology, float* grad_verts, float* grad_coeff,
                          void* workspace, size_t ws_bytes, dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * meshFT in float64: the double-precision dispatch of forward_fourier3d_cpp /
 * backward_fourier3d_cpp (deltamic/cpp/fourier3d_cuda.cpp:27-65; kernels
 * .cu:238-416 for scalar_t = double), i.e. Fourier3dMesh(dtype=torch.float64).
 * Phases xi . v in double and the R1..R5 branches with the reference CPU path's
 * Seps = sqrt(1.19209e-07) (render.py:64-65, strict in R1) -- its CUDA double
 * dispatch uses sqrt(DBL_EPSILON), where the general formula loses the partials
 * to cancellation for phase differences below ~1e-5; every frequency evaluated
 * (band_flags ignored).  Frequencies come from exactly one source:
 *   - a grid band: box and band_index[n_freq] as for dm_meshft_forward (vertices
 *     shifted by box.lo inside, as Fourier3dMesh.forward does); or
 *   - a list: xi_list[n_freq,3] float64 with box NULL (vertices as given, as
 *     forward_fourier3d_cpp takes them).
 * verts[nv,3], faces_coeff[nt] float64; ft_list[n_freq] complex128 (interleaved
 * doubles); grid (grid band only, optional) receives ft * otf at the band's voxels.
 * The backward's cotangent is g[m] = grad_scale * G[m] * (otf ? otf[idx] : 1)
 * with G from grad_list[n_freq] (complex128) or grad_grid (grid band only); it
 * writes grad_verts[nv,3] and, if not NULL, grad_coeff[nt] (float64); topology
 * from dm_topology_build or NULL. */
size_t dm_meshft64_forward_workspace_size(int64_t nv, int64_t nt, int64_t n_freq);
int dm_meshft64_forward(const double* verts, int64_t nv, const int64_t* faces, int64_t nt,
                        const double* faces_coeff, const dm_box* box, const int32_t* band_index,
                        const double* xi_list, int64_t n_freq, const double* otf,
                        double* ft_list, double* grid, void* workspace, size_t ws_bytes,
                        dm_stream_t stream);
size_t dm_meshft64_backward_workspace_size(int64_t nv, int64_t nt, int64_t n_freq);
int dm_meshft64_backward(const double* verts, int64_t nv, const int64_t* faces, int64_t nt,
                         const double* faces_coeff, const dm_box* box,
                         const int32_t* band_index, const double* xi_list, int64_t n_freq,
                         const double* grad_list, const double* grad_grid, const double* otf,
                         double grad_scale, const double* ft_list, const void* topology,
                         double* grad_verts, double* grad_coeff, void* workspace,
                         size_t ws_bytes, dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * Surface + enclosed-volume ("autofluorescence") transform.  Replaces
 * fourier_from_mesh_narrowband_autofluorescence (deltamic/render.py:228-318,
 * pure torch in the reference, differentiated by its autograd):
 *   ft(xi) = sum_k F_k(xi) (2 A_k / sum A + i (regint / regvol) xi.nor_k / |xi|^2)
 * with Heron-equal areas A_k, nor_k = p0 x p1 + p1 x p2 + p2 x p0 and
 * regvol = -sum_k p0 . (p1 x p2) / 6, vertex coordinates AS GIVEN (pass a box
 * with lo = 0 and hi = the box lengths: the reference does not shift the mesh).
 * regint is a DEVICE float.  At xi = 0 (every axis of the grid odd) the
 * reference returns 0/0 = NaN; here the volume term there is its limit -regint.
 * The forward writes ft_list[n_band] and vol_list[n_band] (complex64),
 * vol = i sum_k F_k xi.nor_k / |xi|^2 (-regvol at xi = 0), so that
 * ft = surface part + (regint / regvol) vol; the backward needs both.  The
 * cotangent convention, grad_scale, otf, topology and mirror-symmetric bands are
 * as for dm_meshft_backward; it writes grad_verts[nv,3] and, if not NULL,
 * *grad_regint (DEVICE float). */
size_t dm_meshft_volume_forward_workspace_size(int64_t nv, int64_t nt, int64_t n_band);
int dm_meshft_volume_forward(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                             const float* regint, const dm_box* box, const int32_t* band_index,
                             int64_t n_band, const float* otf, float* ft_list, float* vol_list,
                             float* grid, void* workspace, size_t ws_bytes,
                             dm_stream_t stream);
size_t dm_meshft_volume_backward_workspace_size(int64_t nv, int64_t nt, int64_t n_band);
int dm_meshft_volume_backward(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                              const float* regint, const dm_box* box, const int32_t* band_index,
                              int64_t n_band, const float* grad_list, const float* grad_grid,
                              const float* otf, float grad_scale, const float* ft_list,
                              const float* vol_list, const void* topology, float* grad_verts,
                              float* grad_regint, void* workspace, size_t ws_bytes,
                              dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * Spatial PSF models of deltamic/psf.py: the volume-sized stages (the small
 * per-parameter maps stay with the caller).  All pointers are DEVICE memory.
 *
 * Anisotropic_gaussian_psf (psf.py:628-665): psf[i][j][k] =
 *   exp(-u^T S u / (2 D)) / D, u = (x[i], y[j]), D = eps + (|z[k]| sigma_z)^2,
 * params = {S00, S01, S10, S11, sigma_z, eps} (float32, the reference's operation
 * order); the gradient call writes d loss / d params[6] for grad_psf. */
int dm_aniso_gaussian_psf(const float* params, const float* x, int32_t nx, const float* y,
                          int32_t ny, const float* z, int32_t nz, float* psf, dm_stream_t stream);
size_t dm_aniso_gaussian_psf_grad_workspace_size(int64_t n);
int dm_aniso_gaussian_psf_grad(const float* grad_psf, const float* psf, const float* params,
                               const float* x, int32_t nx, const float* y, int32_t ny,
                               const float* z, int32_t nz, float* grad_params, void* workspace,
                               size_t ws_bytes, dm_stream_t stream);

/* Gibson_Lanni_psf (psf.py:23-154), float64.  The PSF depends on the pixel only
 * through its distance from the lateral centre, so the Fourier-Bessel basis of
 * psf.py:141-143 is formed for the distinct radii u:
 *   basis[u][k] = (s J1(s rm) J0(b rm) rm - b J0(s rm) J1(b rm) rm) / (s s - b b),
 *   s = scaling[k], b = b[u] (= 2 pi radius_u res_lateral NA / wavelength),
 *   rm = *rhomax,
 * with the Bessel values given as tables bessel_s = {J0(s rm)} ++ {J1(s rm)} [2K]
 * and bessel_b = {J0(b rm)} ++ {J1(b rm)} [2U] (the caller's Bessel functions: the
 * amplitude basis @ C cancels large terms of an ill-conditioned least-squares fit,
 * so the basis must use the values the fit used).  dm_radial_basis_grad returns
 * d loss / d scaling[K], d loss / d rhomax[1] and d loss / d b[U]; exact == 0 holds
 * the Bessel values constant, as the reference's autograd does (torch's
 * bessel_j0/j1 have no derivative), exact != 0 differentiates them as well.
 * With the amplitude amp[u][z] = (basis @ C)[u][z] (complex128, interleaved),
 * dm_radial_intensity writes profile[u][z] = |amp|^2, *peak = its maximum and
 * psf[p][z] = profile[pixel_radius[p]][z] / peak for every pixel p = x ny + y; its
 * backward returns d loss / d amp (PyTorch's complex convention), the maximum's
 * gradient shared by every voxel tied with it, as torch's max() does.
 * radius_off[n_radii + 1] / radius_pixels[n_pixels] list the pixels of each
 * radius (CSR, ascending). */
int dm_radial_basis(const double* scaling, int32_t n_basis, const double* rhomax,
                    const double* b, int64_t n_radii, const double* bessel_s,
                    const double* bessel_b, double* basis, dm_stream_t stream);
size_t dm_radial_basis_grad_workspace_size(int64_t n_radii, int32_t n_basis);
int dm_radial_basis_grad(const double* grad_basis, const double* scaling, int32_t n_basis,
                         const double* rhomax, const double* b, int64_t n_radii,
                         const double* bessel_s, const double* bessel_b, int32_t exact,
                         double* grad_scaling, double* grad_rhomax, double* grad_b,
                         void* workspace, size_t ws_bytes, dm_stream_t stream);
size_t dm_radial_intensity_workspace_size(int64_t n_radii, int32_t nz);
int dm_radial_intensity(const double* amp, int64_t n_radii, int32_t nz, const int32_t* pixel_radius,
                        int64_t n_pixels, double* psf, double* profile, double* peak,
                        void* workspace, size_t ws_bytes, dm_stream_t stream);
int dm_radial_intensity_backward(const double* grad_psf, const double* amp, const double* profile,
                                 const double* peak, int64_t n_radii, int32_t nz,
                                 const int32_t* radius_off, const int32_t* radius_pixels,
                                 double* grad_amp, void* workspace, size_t ws_bytes,
                                 dm_stream_t stream);

/* Hanser_psf (psf.py:157-371), float32 / complex64 interleaved.
 * dm_pupil_defocus: pupil[z][x][y] = pupil0[x][y] exp(2 pi i kz[x][y] zr[z])
 * (psf.py:310-314, 336); its backward returns the gradients to pupil0, kz, zr.
 * dm_shifted_intensity: out[x][y][z] = |field[z][x'][y']|^2 with x' = (x - nx/2)
 * mod nx (fftshift over x and y, then the (z, x, y) -> (x, y, z) permutation of
 * psf.py:262-266); its backward returns d loss / d field.  The batched 2-D
 * inverse FFT between them is the caller's (cuFFT).
 * dm_zernike: out[j][i] = Z_{n_j}^{m_j}(r[i], theta[i]), degrees = {n_j, m_j}
 * pairs in HOST memory (n_j <= 10), Noll-normalised, 0 for r > 1 (psf.py:373-548). */
int dm_pupil_defocus(const float* pupil0, const float* kz, const float* zr, int32_t nx,
                     int32_t ny, int32_t nz, float* pupil, dm_stream_t stream);
size_t dm_pupil_defocus_grad_workspace_size(int32_t nx, int32_t ny, int32_t nz);
int dm_pupil_defocus_backward(const float* grad_pupil, const float* pupil0, const float* kz,
                              const float* zr, int32_t nx, int32_t ny, int32_t nz,
                              float* grad_pupil0, float* grad_kz, float* grad_zr,
                              void* workspace, size_t ws_bytes, dm_stream_t stream);
int dm_shifted_intensity(const float* field, int32_t nx, int32_t ny, int32_t nz, float* out,
                         dm_stream_t stream);
int dm_shifted_intensity_backward(const float* field, const float* grad_out, int32_t nx,
                                  int32_t ny, int32_t nz, float* grad_field, dm_stream_t stream);
int dm_zernike(const float* r, const float* theta, int64_t n_points, const int32_t* degrees,
               int32_t n_modes, float* out, dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * Segmentation masks of deltamic/mask_creation.py (float64 vertices [nv,3] and
 * grid; the grid points are numpy.linspace(box.lo[d], box.hi[d], box.shape[d]) per
 * axis, create_coords, mask_creation.py:195-205).
 * dm_membrane_mask (create_semantic_segmentation_mask, :208-222): faces read with
 * face_stride int64 per face (first three = vertex indices) are refined until every
 * edge is at most max_edge (trimesh's subdivide_to_size: four-way splits at the
 * edge midpoints, at most max_depth <= 24 levels, else DM_ERR_SIZE in the
 * workspace's status word), and mask[(ix ny + iy) nz + iz] = 1 at the grid point
 * nearest to each vertex of the refined faces (0 elsewhere).
 * dm_instance_mask (create_instance_segmentation_mask, :225-266): faces [nt,5]
 * (indices, then the labels on either side; a face whose first label is the smaller
 * is flipped, reorder_faces :49-53) split four ways `levels` times
 * (subdivide_with_materials, :60-176); mask[p] = 1 + the label, on grid point p's
 * side of the normal, of the child face whose centroid is nearest to p (ties: the
 * lower child index); the nearest search buckets the child centroids on a uniform
 * grid over the box.  Workspace from dm_mask_workspace_size(nt, levels, box) (box
 * NULL: the membrane mask's 256 bytes); status via dm_device_error. */
size_t dm_mask_workspace_size(int64_t nt, int32_t levels, const dm_box* box);
int dm_membrane_mask(const double* verts, int64_t nv, const int64_t* faces, int64_t nt,
                     int32_t face_stride, const dm_box* box, double max_edge, int32_t max_depth,
                     double* mask, void* workspace, size_t ws_bytes, dm_stream_t stream);
int dm_instance_mask(const double* verts, int64_t nv, const int64_t* faces, int64_t nt,
                     const dm_box* box, int32_t levels, double* mask, void* workspace,
                     size_t ws_bytes, dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * Batches: many meshes ("cells"), each with its own box, grid shape and narrow
 * band, in one launch per stage.  There is no batched counterpart in the
 * reference (one mesh per Fourier3dMesh call, render.py:136-150); the per-cell
 * results equal the single-cell calls above.
 * Concatenation: verts[sum nv,3], faces[sum nt,3] with indices LOCAL to each
 * cell's vertices, faces_coeff[sum nt], band_index[sum n_band] with indices LOCAL
 * to each cell's grid, ft_list[sum n_band]; per-cell grids (otf, spectrum,
 * image) live at grid_offset of one concatenated array. */
typedef struct dm_cell {
  int64_t nv, nt, n_band; /* this cell's mesh and band sizes */
  int64_t grid_offset;    /* first element of its grid in the concatenated grids */
  dm_box box;
} dm_cell;

typedef struct dm_batch {
  int32_t ncells;
  int32_t reserved;
  int64_t nv, nt, n_band, grid_elems;           /* totals */
  int64_t fwd_workspace, bwd_workspace;         /* workspace bytes for the calls below */
  int64_t topology_bytes, image_workspace;
  int64_t plan[12];                             /* launch sizes (opaque) */
  const void* cells;                            /* device copy of the cell plan */
} dm_batch;

/* Bytes of the device buffer that holds the plan of ``ncells`` cells. */
size_t dm_batch_desc_size(int ncells);
/* Plans the batch, uploads the cell plan into ``desc`` (device, desc_bytes) and
 * fills *out.  Synchronous (waits for the upload): call it outside stream capture,
 * once per set of meshes and bands. */
int dm_batch_plan(const dm_cell* cells, int ncells, void* desc, size_t desc_bytes,
                  dm_batch* out, dm_stream_t stream);
int dm_batched_topology_build(const dm_batch* batch, const int64_t* faces, void* topology,
                              size_t topo_bytes, dm_stream_t stream);
int dm_batched_meshft_forward(const dm_batch* batch, const float* verts, const int64_t* faces,
                              const float* faces_coeff, const int32_t* band_index,
                              const float* otf, float* ft_list, float* grid, void* workspace,
                              size_t ws_bytes, dm_stream_t stream);
int dm_batched_meshft_backward(const dm_batch* batch, const float* verts, const int64_t* faces,
                               const float* faces_coeff, const int32_t* band_index,
                               const float* grad_list, const float* grad_grid, const float* otf,
                               float grad_scale, const float* ft_list, const void* topology,
                               float* grad_verts, float* grad_coeff, float* grad_otf_band,
                               void* workspace, size_t ws_bytes, dm_stream_t stream);
/* dm_image_loss per cell image (loss[ncells], each normalised by its own min/max). */
int dm_batched_image_loss(const dm_batch* batch, const float* z, int kind, const float* target,
                          float contrast, float* image, float* loss, float* grad_z,
                          void* workspace, size_t ws_bytes, dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * Gaussian OTF.  Replaces generate_gaussian_psf (deltamic/psf.py:15-20):
 *   otf[i,j,k] = exp(-(x^T S x)/2),  x = (xi0[i], xi1[j], xi2[k]),
 * S = sigma[3,3] (DEVICE float32, row-major, as the torch parameter), on the
 * outer grid of the three DEVICE float32 axes (Fourier3dMesh.xi0/xi1/xi2),
 * evaluated with the reference expression's float32 operation order. */
int dm_gaussian_otf(const float* sigma, const float* xi0, int32_t n0, const float* xi1,
                    int32_t n1, const float* xi2, int32_t n2, float* otf, dm_stream_t stream);

/* d loss / d sigma for that OTF: grad_sigma[i*3+j] = sum over voxels of
 * grad_otf * otf * (-x_i x_j / 2).  Dense form (band_index NULL: grad_otf[n0 n1 n2])
 * or band form (grad_otf[n_band] holds the values at voxels band_index[m]). */
size_t dm_gaussian_otf_grad_workspace_size(int64_t n);
int dm_gaussian_otf_sigma_grad(const float* grad_otf, const int32_t* band_index, int64_t n_band,
                               const float* otf, const float* xi0, int32_t n0, const float* xi1,
                               int32_t n1, const float* xi2, int32_t n2, float* grad_sigma,
                               void* workspace, size_t ws_bytes, dm_stream_t stream);

/* The same two calls in float64 (generate_gaussian_psf on float64 sigma and axes,
 * Fourier3dMesh(dtype=torch.float64)): the reference expression's operation
 * order in double; workspace from dm_gaussian_otf_grad_workspace_size. */
int dm_gaussian_otf64(const double* sigma, const double* xi0, int32_t n0, const double* xi1,
                      int32_t n1, const double* xi2, int32_t n2, double* otf,
                      dm_stream_t stream);
int dm_gaussian_otf64_sigma_grad(const double* grad_otf, const int32_t* band_index,
                                 int64_t n_band, const double* otf, const double* xi0, int32_t n0,
                                 const double* xi1, int32_t n1, const double* xi2, int32_t n2,
                                 double* grad_sigma, void* workspace, size_t ws_bytes,
                                 dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * Fused image stage on the inverse FFT z = ifftn(ftmesh * OTF) (complex64[n]):
 * image = |z| (render_image_from_ftmesh, render.py:177-180), normalised by
 * normalize_tensor (render.py:5-6) with ``contrast``, then the loss
 *   kind 0: sum(normalised image)
 *   kind 1: mean((normalised image - target)^2)
 * Writes *loss (DEVICE float), optionally image[n] = |z|, and, if grad_z is not
 * NULL, dL/dz in PyTorch's complex convention (ties of the min / max share
 * their gradient evenly, as torch's full min/max reductions do). */
size_t dm_image_loss_workspace_size(int64_t n);
int dm_image_loss(const float* z, int64_t n, int kind, const float* target, float contrast,
                  float* image, float* loss, float* grad_z, void* workspace, size_t ws_bytes,
                  dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * normalize_tensor (render.py:5-6) of a real array t[n] (any shape, contiguous):
 *   out = ((t - min t) / (max t - min t) + c) / (1 + c),   c = contrast
 * in the operation order of the eager expression on a CUDA tensor (the scalar
 * division as a product with its reciprocal).  min / max propagate NaN.
 * dm_normalize writes stats[2] = (min, max) (DEVICE) and, if out is not NULL,
 * out[n].  dm_normalize_backward takes those stats and dL/dout and writes dL/dt,
 * the min / max terms shared evenly by tied elements (torch's rule for full
 * min() / max() reductions).  Deterministic; 2 launches each. */
size_t dm_normalize_workspace_size(int64_t n);
int dm_normalize(const float* t, int64_t n, double contrast, float* out, float* stats,
                 void* workspace, size_t ws_bytes, dm_stream_t stream);
int dm_normalize_backward(const float* t, const float* grad_out, int64_t n, double contrast,
                          const float* stats, float* grad_t, void* workspace, size_t ws_bytes,
                          dm_stream_t stream);
int dm_normalize64(const double* t, int64_t n, double contrast, double* out, double* stats,
                   void* workspace, size_t ws_bytes, dm_stream_t stream);
int dm_normalize64_backward(const double* t, const double* grad_out, int64_t n, double contrast,
                            const double* stats, double* grad_t, void* workspace,
                            size_t ws_bytes, dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * Band-box render: the chain render_image_from_ftmesh -> normalize_tensor ->
 * loss of the reference fitting loop (render.py:177-180, render.py:5-6,
 * Examples/Gradient_Descent.ipynb cell 2) and its backward to the spectrum,
 * for a spectrum that is zero outside the narrow band.  Replaces the dense
 * ifftn / image loss / fftn sequence (torch.fft on the dense grid of
 * cuda_class.py:28-29) by separable DFTs pruned to the band's bounding box.
 *
 * dm_band_bounds writes bounds[6] (DEVICE int32) = per-axis smallest band index
 * (lo0, lo1, lo2) then largest (hi0, hi1, hi2); the other calls take the same six
 * numbers from HOST memory.  dm_render_loss_bandbox_supported says whether this
 * build serves a box (band extent along axis 2 at most 32 and the line tiles
 * within shared memory); otherwise the call returns DM_ERR_UNSUPPORTED and the
 * dense path applies.
 * dm_render_loss_bandbox takes ft_list[n_band] (complex64, the band's meshFT as
 * dm_meshft_forward returns it) and the OTF, forms S = ft * OTF on the band and
 * z = ifftn(S) over the whole box, then the loss of dm_image_loss (same kinds,
 * contrast and min / max tie rule).  Writes *loss (DEVICE float), optionally
 * image[n] = |z|, and, if grad_list is not NULL, grad_list[n_band] = fftn(dL/dz)
 * at the band voxels (complex64): the cotangent dm_meshft_backward takes as
 * grad_list with otf and grad_scale = 1/n.  Deterministic.
 * kind 2 renders without a loss: ``target`` then holds a cotangent dL/dimage[n]
 * of the image |z| itself (no normalisation; *loss is written as 0), and
 * grad_list receives fftn(dL/dz) at the band voxels for it -- the adjoint of
 * render_image_from_ftmesh (render.py:177-180) for a band-limited spectrum.
 * With kind 2 and grad_list NULL the call only renders (image, *loss = 0) and
 * target may be NULL. */
int dm_band_bounds(const int32_t* band_index, int64_t n_band, const dm_box* box,
                   int32_t* bounds, dm_stream_t stream);
int dm_render_loss_bandbox_supported(const dm_box* box, const int32_t bounds[6]);
size_t dm_render_loss_bandbox_workspace_size(const dm_box* box, const int32_t bounds[6]);
int dm_render_loss_bandbox(const float* ft_list, const int32_t* band_index, int64_t n_band,
                           const dm_box* box, const int32_t bounds[6], const float* otf,
                           int kind, const float* target, float contrast, float* loss,
                           float* grad_list, float* image, void* workspace, size_t ws_bytes,
                           dm_stream_t stream);

/* Band-box render + loss for the cells of a batch (each cell's box, band and
 * loss as dm_render_loss_bandbox alone; kinds 0 and 1).  The plan (host,
 * synchronous, outside stream capture) takes the cells (box, n_band,
 * grid_offset of dm_cell) and their band bounds (HOST int32 [ncells][6], as
 * dm_band_bounds writes them); it owns ``workspace`` (its size from
 * dm_bandbox_batch_workspace_size, DM_ERR_UNSUPPORTED if a cell's box is not
 * served) and uploads its tables into ``desc`` (dm_bandbox_batch_desc_size).
 * dm_bandbox_batch_render_loss takes the concatenated band lists (ft_list,
 * band_index with cell-local voxel indices) and concatenated grids (otf, target,
 * image at each cell's grid_offset), writes loss[ncells] (DEVICE) and, if
 * grad_list is not NULL, grad_list = fftn(dL/dz) / n_cell at each cell's band
 * voxels: dL/dS, the cotangent dm_batched_meshft_backward takes with otf and
 * grad_scale 1.  One launch per stage for all cells (the two line passes: one
 * per distinct line-tile shape).  dm_bandbox_batch_device_error reads and clears
 * the cells' status words (synchronous). */
typedef struct dm_bandbox_batch {
  int32_t ncells;
  int32_t reserved;
  int64_t workspace_bytes;
  int64_t plan[128]; /* launch sizes (opaque) */
  const void* cells; /* device copy of the plan */
  void* workspace;
} dm_bandbox_batch;

size_t dm_bandbox_batch_desc_size(int ncells);
int dm_bandbox_batch_workspace_size(const dm_cell* cells, const int32_t* bounds, int ncells,
                                    size_t* bytes);
int dm_bandbox_batch_plan(const dm_cell* cells, const int32_t* bounds, int ncells, void* desc,
                          size_t desc_bytes, void* workspace, size_t ws_bytes,
                          dm_bandbox_batch* out, dm_stream_t stream);
int dm_bandbox_batch_render_loss(const dm_bandbox_batch* bb, const float* ft_list,
                                 const int32_t* band_index, const float* otf, int kind,
                                 const float* target, float contrast, float* loss,
                                 float* grad_list, float* image, dm_stream_t stream);
int dm_bandbox_batch_device_error(const dm_bandbox_batch* bb, int* out_flags,
                                  dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * 3x3x3 stride-2 padding-1 3D convolution with bias and GELU, for the learned
 * initialiser's encoder (no counterpart in the reference).  Channels-last BF16
 * tensors (uint16 storage): x[B,D,H,W,Ci], w[Kp,Co] with row k = ((kd*3+kh)*3+kw)*Ci
 * + ci and Kp = 27*Ci rounded up to 32 (padding rows zero); Co in {16,32,64,128},
 * Ci <= 128, B*D*H*W*max(Ci, Co) < 2^31; output (D+1)/2 x (H+1)/2 x (W+1)/2.  Implicit GEMMs on the fifth-
 * generation tensor cores (tcgen05 MMAs, FP32 accumulators in tensor memory).
 * Forward writes pre[.., Co] (FP32 pre-activation) and act = GELU(pre) (BF16).
 * Backward takes dact = dL/dact (FP32) and writes dw[Kp,Co], db[Co] and, if
 * dx != NULL, dx = dL/dx (FP32); deterministic (no atomics).
 * dm_conv3d_s2_device_error reads and clears the kernels' status word
 * (DM_ERR_TIMEOUT: a bounded wait for the tensor cores gave up); synchronous. */
size_t dm_conv3d_s2_workspace_size(int B, int D, int H, int W, int Ci, int Co);
int dm_conv3d_s2_forward(const uint16_t* x, int B, int D, int H, int W, int Ci, const uint16_t* w,
                         const float* bias, int Co, float* pre, uint16_t* act,
                         dm_stream_t stream);
/* The forward with a workspace (its size from the query): when the row tiles alone
 * would leave SMs idle (small layers), the reduction is split across blocks and the
 * FP32 partials are added in split order before the bias and GELU (deterministic). */
size_t dm_conv3d_s2_forward_workspace_size(int B, int D, int H, int W, int Ci, int Co);
int dm_conv3d_s2_forward_ws(const uint16_t* x, int B, int D, int H, int W, int Ci,
                            const uint16_t* w, const float* bias, int Co, float* pre,
                            uint16_t* act, void* workspace, size_t ws_bytes, dm_stream_t stream);
int dm_conv3d_s2_device_error(int* out_flags, dm_stream_t stream);
int dm_conv3d_s2_backward(const uint16_t* x, int B, int D, int H, int W, int Ci,
                          const uint16_t* w, int Co, const float* pre, const float* dact,
                          float* dx, float* dw, float* db, void* workspace, size_t ws_bytes,
                          dm_stream_t stream);
/* The same with dact and dx in BF16 (the dtype of the activations they belong
 * to), as an autograd chain of these layers passes them: no FP32 round trip. */
int dm_conv3d_s2_backward_bf16(const uint16_t* x, int B, int D, int H, int W, int Ci,
                               const uint16_t* w, int Co, const float* pre, const uint16_t* dact,
                               uint16_t* dx, float* dw, float* db, void* workspace,
                               size_t ws_bytes, dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * Occupancy of a closed mesh (for the volumetric IoU of a fit; no counterpart in
 * the reference, whose label tooling uses a KD-tree on the host,
 * mask_creation.py:210-224).  occupancy[n0,n1,n2] (uint8 0/1) at the image sample
 * positions lo + (i,j,k) L/n, by ray parity along the third axis.  ``status``
 * (DEVICE int, may be NULL) receives DM_ERR_BAD_INDEX for face indices outside
 * [0, nv) and DM_ERR_SIZE for a column with more than 64 crossings. */
int dm_voxelize(const float* verts, int64_t nv, const int64_t* faces, int64_t nt,
                const dm_box* box, uint8_t* occupancy, int* status, dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * Adam step (torch.optim.Adam semantics, no weight decay) on a float32 array;
 * ``step`` is a DEVICE int64 counter that the call increments (1-based after). */
int dm_adam_step(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, int64_t n,
                 float lr, float beta1, float beta2, float eps, int64_t* step,
                 dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * OTF of a spatial PSF (the notebook's OTF = |fftshift(fftn(PSF))|,
 * Examples/Gradient_Descent.ipynb cell 2, PSF from psf.py:551-587), around the
 * caller's 3-D FFT: dm_otf_from_spectrum writes otf[k] = |spectrum[k - n/2 mod n]|
 * (fftshift and |.| fused); dm_otf_from_spectrum_backward writes
 * grad_spectrum[j] = grad_otf[j + n/2 mod n] * spectrum[j] / |spectrum[j]|
 * (0 where the spectrum is 0).  spectrum / grad_spectrum complex64 [n0,n1,n2]. */
int dm_otf_from_spectrum(const float* spectrum, int32_t n0, int32_t n1, int32_t n2, float* otf,
                         dm_stream_t stream);
int dm_otf_from_spectrum_backward(const float* spectrum, const float* grad_otf, int32_t n0,
                                  int32_t n1, int32_t n2, float* grad_spectrum,
                                  dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * Preconditioned fit (the reference notebook's gradient preconditioning,
 * Examples/Gradient_Descent.ipynb cell 2: Verts.grad = solve(M@M, Verts.grad),
 * M = I + lambda L from largesteps' compute_matrix; optimize.py:207-212 forms the
 * same operator densely as inv(M) @ inv(M)).
 * dm_precond_apply: out[nv,3] = P grad[nv,3] for a dense P[nv, ldp] (float32,
 * row-major, ldp a multiple of 4 with zero padding, 16-byte aligned); out must
 * not alias grad.
 * dm_vector_adam_step: VectorAdam of optimize.py:215-258 (axis -1): per-vertex
 * second moment exp_avg_norm_sq[nv] of the squared gradient norm; ``step`` is a
 * DEVICE int64 counter that the call increments. */
int dm_precond_apply(const float* P, int64_t nv, int64_t ldp, const float* grad, float* out,
                     dm_stream_t stream);
/* (M M)^-1 grad without forming the operator: two Chebyshev solves with
 * M = I + lambda L for the eigenvalue interval [lo, hi] of M (lo > 0), ``iters``
 * iterations each (one launch per iteration).  L from CSR neighbour lists rowp[nv+1],
 * col[] (DEVICE int32: row i lists the vertices sharing an edge with i, so L = D - A
 * of the uniform Laplacian); grad, out [nv][3]; work: 12 nv floats (DEVICE). */
int dm_precond_chebyshev(const int32_t* rowp, const int32_t* col, int64_t nv, float lambda,
                         double lo, double hi, int iters, const float* grad, float* out,
                         float* work, dm_stream_t stream);
int dm_vector_adam_step(float* param, const float* grad, float* exp_avg, float* exp_avg_norm_sq,
                        int64_t nv, float lr, float beta1, float beta2, float eps, int64_t* step,
                        dm_stream_t stream);

/* ---------------------------------------------------------------------------
 * Instrumentation (no counterpart in the reference, which has no profiling).
 * dm_launch_count: kernels this library has launched in the process (host-side
 * count; graph replays are not counted).
 * dm_profile_enable: when on, every launch of the main meshFT forward (kernel 0)
 * or adjoint (kernel 1) kernel is bracketed by CUDA events on its stream (up to
 * 512 per kernel between reads).  Not for use inside stream capture.
 * dm_profile_read: synchronises those events and returns their count and total
 * milliseconds, then clears them. */
long long dm_launch_count(void);

/* Tile-shape variants of the meshFT forward and adjoint kernels (no counterpart in
 * the reference).  Process-wide; a plan, workspace size and launch use the
 * variants current when they are made, so re-query workspace sizes after a
 * change and do not change variants between a workspace query and its call.
 * The autotuner (deltamic_b200.autotune) picks them per size class. */
int dm_set_variants(int fwd, int bwd);
int dm_get_variants(int* fwd, int* bwd, int* n_fwd, int* n_bwd);

/* Self-test of the library's bounded device waits (no counterpart in the
 * reference): one block waits on an mbarrier that nothing completes -- with the
 * spinning wait (mode 0, at most limit <= 2^22 polls) or the sleeping wait of the
 * persistent kernels (mode 1, at most limit <= 2^16 tries of 20 us) -- gives up,
 * ORs DM_ERR_TIMEOUT into *status (DEVICE int, caller-zeroed) and returns, leaving
 * the context usable.  Shows that a wait that never completes ends the kernel
 * with a status instead of hanging it. */
int dm_selftest_bounded_wait(int mode, uint32_t limit, int* status, dm_stream_t stream);

/* Throughput probe (no counterpart in the reference): times ``iters`` rounds of
 * 8 independent FP32 FMA chains (kind 0), MUFU sin.approx chains (kind 1) or
 * paired FP32 FMA chains (kind 2, sm_100 FFMA2) per thread over the whole GPU and
 * returns FMAs (kinds 0, 2) or sines (kind 1) per second.  Synchronous; these
 * are the roofline denominators for the FP32/MUFU-bound meshFT kernels. */
int dm_peak_probe(int kind, int iters, double* ops_per_s, dm_stream_t stream);
int dm_profile_enable(int enable);
int dm_profile_read(int kernel, int* count, float* total_ms);

#ifdef __cplusplus
}
#endif

#endif /* DELTAMIC_B200_H_ */
