"""``MeshFTCUDA``: the reference's autograd entry point (cuda_class.py:10-41) with
its signature, on this library's kernels.

``MeshFTCUDA.apply(Verts, Faces, Faces_coeff, xi0, xi1, xi2, Filter,
narrowband_thresh)`` returns the dense complex spectrum on the grid of the three
centred frequency axes, zero outside ``Filter > narrowband_thresh``, for the vertex
coordinates as given (the phase of every vertex is ``xi . v``).  As in the
reference, only ``Verts`` receives a gradient.  The axes must be the centred grids
``(2k - (n - 1)) pi / L`` that ``compute_spatial_frequency_grid`` makes (the
kernels evaluate the phases in exact fixed point on that grid); other axes raise
``ValueError``.  A float64 ``Verts`` is evaluated in float32 and returns complex128,
as ``Fourier3dMesh(dtype=float64)`` does.
"""
from __future__ import annotations

import numpy as np
import torch

from . import ops
from .render import _axis_length

__all__ = ["MeshFTCUDA"]

_BANDS: dict = {}


class MeshFTCUDA:
    """Drop-in for ``deltamic.cuda_class.MeshFTCUDA`` (use ``MeshFTCUDA.apply``)."""

    @staticmethod
    def apply(Verts, Faces, Faces_coeff, xi0, xi1, xi2, Filter, narrowband_thresh):
        if Verts.dtype not in (torch.float, torch.double):
            raise TypeError("Mesh FT not implemented for " + str(Verts.dtype))
        shape = (int(xi0.numel()), int(xi1.numel()), int(xi2.numel()))
        if tuple(Filter.shape) != shape:
            raise ValueError(f"Filter shape {tuple(Filter.shape)} does not match the axes "
                             f"{shape}")
        L = [_axis_length(x) for x in (xi0, xi1, xi2)]
        grid = ops.FreqGrid(np.array([[0.0, L[0]], [0.0, L[1]], [0.0, L[2]]]), shape)
        thr = float(narrowband_thresh)
        key = (Filter.data_ptr(), Filter._version, shape, thr)
        hit = _BANDS.get(id(Filter))
        if hit is not None and hit[0] == key:
            band = hit[1]
        else:
            band = ops.narrowband(Filter.detach().float().contiguous(), thr)
            _BANDS.clear()
            _BANDS[id(Filter)] = (key, band)
        f64 = Verts.dtype == torch.float64
        coeff = Faces_coeff.detach().float()  # the reference returns no coefficient gradient
        out = ops.meshft(Verts.float() if f64 else Verts, Faces, coeff, grid, band)
        return out.to(torch.complex128) if f64 else out
