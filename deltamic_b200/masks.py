"""Segmentation masks of ``deltamic/mask_creation.py`` on the GPU kernels of
``masks.cu``, with the reference's small numpy helpers.

* ``create_semantic_segmentation_mask(verts, faces, box_shape, box_size)``
  (mask_creation.py:208-222): the membrane mask, returned FLAT (nx*ny*nz, float64)
  as the reference returns it (its ``reshape`` result is discarded);
* ``create_instance_segmentation_mask(verts, faces, box_shape, box_size)``
  (:225-266): faces [nt,5] with the labels on either side; the label mask
  (float64, box_shape), labels + 1;
* ``create_coords``, ``compute_box_size`` (the per-axis box of this module,
  :186-192), ``compute_max_size_edges`` (kept as the reference computes it: the
  norm of the stacked edge vectors b-a, c-b, c-b), ``reorder_faces``,
  ``create_voxel_centroids``.

Numpy inputs give numpy results (drop-in); the work runs on ``device``.  The label
mask's nearest-centroid search buckets the child faces' centroids on a uniform grid
(exact; ties to the lower child index).  The
refinement (trimesh's ``subdivide_to_size`` / the reference's
``subdivide_with_materials``) happens inside the kernels, face by face.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native as N

__all__ = ["create_semantic_segmentation_mask", "create_instance_segmentation_mask",
           "create_coords", "compute_box_size", "compute_max_size_edges", "reorder_faces",
           "create_voxel_centroids"]


def compute_max_size_edges(Verts, Faces):
    P = np.asarray(Verts)[np.asarray(Faces)[:, [0, 1, 2]]]
    E = np.hstack((P[:, 1] - P[:, 0], P[:, 2] - P[:, 1], P[:, 2] - P[:, 1]))
    return np.amax(np.linalg.norm(E, axis=1))


def reorder_faces(Faces):
    """Faces whose first label is the smaller get their orientation and labels
    swapped (in place, as the reference)."""
    for i, face in enumerate(Faces):
        if face[3] < face[4]:
            Faces[i] = Faces[i][[0, 2, 1, 4, 3]]
    return Faces


def create_voxel_centroids(nx, ny, nz):
    XV = np.linspace(0.5, nx - 0.5, nx - 1)
    YV = np.linspace(0.5, ny - 0.5, ny - 1)
    ZV = np.linspace(0.5, nz - 0.5, nz - 1)
    gx, gy, gz = np.meshgrid(XV, YV, ZV, indexing="ij")
    return np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)


def compute_box_size(verts, offset=0.1):
    extent = verts.max(axis=0) - verts.min(axis=0)
    box = np.zeros((3, 2))
    box[:, 1] = verts.max(axis=0) + extent * offset / 2
    box[:, 0] = verts.min(axis=0) - extent * offset / 2
    return box


def create_coords(box_shape, box_size):
    nx, ny, nz = (int(v) for v in box_shape)
    X = np.linspace(box_size[0, 0], box_size[0, 1], nx)
    Y = np.linspace(box_size[1, 0], box_size[1, 1], ny)
    Z = np.linspace(box_size[2, 0], box_size[2, 1], nz)
    gx, gy, gz = np.meshgrid(X, Y, Z, indexing="ij")
    return np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)


def _box(box_shape, box_size):
    b = np.asarray(torch.as_tensor(box_size).detach().cpu().double().numpy(), np.float64)
    shape = [int(v) for v in np.asarray(box_shape).ravel()]
    return N.make_box(b, shape), b, np.array(shape)


def _dev(x, dtype, device):
    return torch.as_tensor(np.ascontiguousarray(x) if isinstance(x, np.ndarray) else x,
                           dtype=dtype, device=device).contiguous()


def _status(ws, device):
    flags = ctypes.c_int(0)
    N.check(N.lib().dm_device_error(N.ptr(ws), ctypes.byref(flags), N.stream_ptr(device)),
            "dm_device_error")
    return flags.value


def create_semantic_segmentation_mask(verts, faces, box_shape, box_size, device="cuda"):
    numpy_in = not isinstance(verts, torch.Tensor)
    cbox, b, shape = _box(box_shape, box_size)
    dmax = float(np.amin((b[:, 1] - b[:, 0]) / shape))
    V = _dev(verts, torch.float64, device)
    F = _dev(faces, torch.int64, device)
    if F.dim() != 2 or F.shape[1] < 3:
        raise ValueError("faces must have shape [nt, >=3]")
    nt = F.shape[0]
    if nt:
        P = V[F[:, :3]]
        e = torch.cat([P[:, 1] - P[:, 0], P[:, 2] - P[:, 1], P[:, 0] - P[:, 2]])
        longest = float(torch.linalg.norm(e, dim=1).max())
        max_iter = max(int(np.ceil(np.log2(longest / dmax))), 0) * 2 + 1
    else:
        max_iter = 0
    out = torch.empty(int(np.prod(shape)), dtype=torch.float64, device=V.device)
    lib = N.lib()
    ws = N.WORKSPACES.get("mask", 256, V.device)
    ws.zero_()
    N.check(lib.dm_membrane_mask(N.ptr(V), V.shape[0], N.ptr(F), nt, F.shape[1],
                                 ctypes.byref(cbox), dmax, min(max_iter, 24), N.ptr(out),
                                 N.ptr(ws), ws.numel(), N.stream_ptr(V.device)),
            "dm_membrane_mask")
    flags = _status(ws, V.device)
    if flags:
        raise ValueError("max_iter exceeded!" if flags & N.DM_ERR_SIZE else
                         f"membrane mask: {N.lib().dm_status_string(flags).decode()}")
    return out.cpu().numpy() if numpy_in else out


def create_instance_segmentation_mask(verts, faces, box_shape, box_size, device="cuda"):
    numpy_in = not isinstance(verts, torch.Tensor)
    fz = np.asarray(faces.detach().cpu() if isinstance(faces, torch.Tensor) else faces)
    assert fz.shape[1] == 5
    cbox, b, shape = _box(box_shape, box_size)
    dmax = float(np.amin((b[:, 1] - b[:, 0]) / shape))
    vz = np.asarray(verts.detach().cpu() if isinstance(verts, torch.Tensor) else verts,
                    np.float64)
    longest = compute_max_size_edges(vz, fz)
    levels = min(max(int(np.ceil(np.log2(longest / dmax))) - 2, 0), 3)
    V = _dev(vz, torch.float64, device)
    F = _dev(fz.astype(np.int64), torch.int64, device)
    lib = N.lib()
    nbytes = lib.dm_mask_workspace_size(F.shape[0], levels, ctypes.byref(cbox))
    ws = torch.zeros(max(nbytes, 256), dtype=torch.uint8, device=V.device)
    out = torch.empty(tuple(int(s) for s in shape), dtype=torch.float64, device=V.device)
    N.check(lib.dm_instance_mask(N.ptr(V), V.shape[0], N.ptr(F), F.shape[0], ctypes.byref(cbox),
                                 levels, N.ptr(out), N.ptr(ws), ws.numel(),
                                 N.stream_ptr(V.device)), "dm_instance_mask")
    flags = _status(ws, V.device)
    if flags:
        raise ValueError(f"instance mask: {N.lib().dm_status_string(flags).decode()}")
    return out.cpu().numpy() if numpy_in else out
