"""deltamic_b200: the deltaMic render-and-fit hot path on NVIDIA B200 (sm_100a).

Drop-in names of the reference package (``from deltamic import ...``):
``Fourier3dMesh``, ``generate_gaussian_psf``, ``generate_gaussian_psf_from_sigma``,
``render_image_from_ftmesh``, ``normalize_tensor``, ``compute_box_size``,
``compute_spatial_frequency_grid``, ``center_verts_in_box``,
``fourier_from_mesh_narrowband_autofluorescence``, the PSF modules, the mask and
mesh-file helpers; by module: ``deltamic_b200.cuda_class.MeshFTCUDA``,
``deltamic_b200.optimize.{compute_precondition_matrix, VectorAdam}``.

Beyond the reference: ``MeshRenderer`` (fused render + loss + adjoint),
``fit_mesh`` / ``FitStep`` (Adam fitting loop, CUDA-graph captured), and the
synthetic mesh generators in ``deltamic_b200.mesh``.

All compute runs in hand-written CUDA kernels of ``lib/libdeltamic_b200.so``
behind a C ABI (``include/deltamic_b200.h``); there is no CPU fallback.
"""
from .psf import (Anisotropic_gaussian_psf, Gaussian_psf, Gaussian_psf_logsigma,
                  Gibson_Lanni_psf, Hanser_psf, generate_gaussian_psf,
                  generate_gaussian_psf_from_sigma, noll2degrees, otf_from_psf, zernike)
from .render import (Fourier3dMesh, center_verts_in_box, compute_box_size,
                     compute_spatial_frequency_grid, compute_volume_manifold,
                     fourier_from_mesh_narrowband_autofluorescence,
                     get_internal_triangle_and_mesh_areas,
                     get_internal_triangle_and_mesh_areas_and_normals,
                     get_internal_triangle_and_mesh_areas_with_coeff, normalize_tensor,
                     render_image_from_ftmesh)
from .pipeline import MeshRenderer
from . import cuda_class, masks, mesh_io, optimize
from .cuda_class import MeshFTCUDA
from .optimize import VectorAdam, compute_precondition_matrix
from .masks import create_instance_segmentation_mask, create_semantic_segmentation_mask
from .mesh_io import create_initial_mesh_from_points_mm, read_obj, read_rec, write_obj, write_rec

__all__ = [
    "Fourier3dMesh", "generate_gaussian_psf", "generate_gaussian_psf_from_sigma",
    "render_image_from_ftmesh", "normalize_tensor", "compute_box_size",
    "compute_spatial_frequency_grid", "center_verts_in_box", "MeshRenderer", "Gaussian_psf",
    "otf_from_psf", "fourier_from_mesh_narrowband_autofluorescence", "Gaussian_psf_logsigma",
    "Anisotropic_gaussian_psf", "Gibson_Lanni_psf", "Hanser_psf", "zernike", "noll2degrees",
    "get_internal_triangle_and_mesh_areas", "get_internal_triangle_and_mesh_areas_and_normals",
    "get_internal_triangle_and_mesh_areas_with_coeff", "MeshFTCUDA", "VectorAdam",
    "compute_precondition_matrix", "compute_volume_manifold", "create_semantic_segmentation_mask",
    "create_instance_segmentation_mask", "create_initial_mesh_from_points_mm", "read_obj",
    "write_obj", "read_rec", "write_rec",
]
