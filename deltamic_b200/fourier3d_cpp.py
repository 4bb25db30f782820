"""The reference's native module under its own names: ``forward_fourier3d_cpp`` and
``backward_fourier3d_cpp`` (deltamic/cpp/fourier3d_cuda.cpp:27-65, bound at
:112-115 as ``deltamic.fourier3d_cpp``), on this library's kernels.

* ``forward_fourier3d_cpp(Verts, Faces, Faces_coeff, xi_list)`` -> ``ftmesh_list``
  [N] complex64 (float32 inputs) or complex128 (float64 inputs): the analytic
  transform of the mesh (vertex coordinates as given) at every row of
  ``xi_list`` [N, 3], ``(2/M) sum_k A_k c_k F_k(xi)``.
* ``backward_fourier3d_cpp(Verts, Faces, Faces_coeff, grad_output_list,
  ftmesh_list, xi_list)`` -> ``gradVerts`` [nv, 3] for the cotangent
  ``grad_output_list`` (PyTorch's convention for complex outputs).

As in the reference every tensor must be a contiguous CUDA tensor (else
``RuntimeError``); float32 inputs run the split-phase float32 kernels (any
frequencies, on a grid or not), float64 inputs the float64 kernels (the
reference's double arithmetic).  Verts, Faces_coeff and xi_list share one dtype,
Faces is int64.  There is no CPU path.
"""
from __future__ import annotations

import torch

from . import ops

__all__ = ["forward_fourier3d_cpp", "backward_fourier3d_cpp"]


def _check_input(x, name):
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if not x.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")


def _check_mesh(Verts, Faces, Faces_coeff, xi_list):
    for x, n in ((Verts, "mesh_vertices"), (Faces, "mesh_faces"), (Faces_coeff, "faces_coeff"),
                 (xi_list, "xi_list")):
        _check_input(x, n)
    dt = Verts.dtype
    if dt not in (torch.float32, torch.float64):
        raise RuntimeError(f"Mesh FT not implemented for {dt}")
    if Faces_coeff.dtype != dt or xi_list.dtype != dt:
        raise RuntimeError("mesh_vertices, faces_coeff and xi_list must share one dtype")
    if Faces.dtype != torch.int64:
        raise RuntimeError("mesh_faces must be int64")
    if Verts.dim() != 2 or Verts.shape[1] != 3 or Faces.dim() != 2 or Faces.shape[1] != 3:
        raise RuntimeError("mesh_vertices and mesh_faces must have shape [n, 3]")
    if xi_list.dim() != 2 or xi_list.shape[1] != 3:
        raise RuntimeError("xi_list must have shape [N, 3]")
    if Faces_coeff.shape != (Faces.shape[0],):
        raise RuntimeError("faces_coeff must have shape [n_faces]")
    return dt


def forward_fourier3d_cpp(Verts, Faces, Faces_coeff, xi_list):
    dt = _check_mesh(Verts, Faces, Faces_coeff, xi_list)
    Verts, Faces_coeff, xi_list = Verts.detach(), Faces_coeff.detach(), xi_list.detach()
    if dt == torch.float64:
        return ops.meshft64_list(Verts, Faces, Faces_coeff, xi_list=xi_list)
    return ops.meshft_xi_list(Verts, Faces, Faces_coeff, xi_list)


def backward_fourier3d_cpp(Verts, Faces, Faces_coeff, grad_output_list, ftmesh_list, xi_list):
    dt = _check_mesh(Verts, Faces, Faces_coeff, xi_list)
    _check_input(grad_output_list, "grad_output_list")
    _check_input(ftmesh_list, "ftmesh_list")
    ct = torch.complex128 if dt == torch.float64 else torch.complex64
    n = xi_list.shape[0]
    for x, name in ((grad_output_list, "grad_output_list"), (ftmesh_list, "ftmesh_list")):
        if x.dtype != ct or x.shape != (n,):
            raise RuntimeError(f"{name} must be {ct} of shape [{n}]")
    Verts, Faces_coeff, xi_list = Verts.detach(), Faces_coeff.detach(), xi_list.detach()
    if dt == torch.float64:
        gv, _ = ops.meshft64_backward_list(Verts, Faces, Faces_coeff, ftmesh_list.detach(),
                                           xi_list=xi_list, grad_list=grad_output_list.detach(),
                                           want_coeff=False)
        return gv
    gv, _ = ops.meshft_xi_backward_list(Verts, Faces, Faces_coeff, xi_list,
                                        grad_output_list.detach(), ftmesh_list.detach(),
                                        want_coeff=False)
    return gv

