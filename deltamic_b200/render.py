"""Drop-in rendering API of deltaMic (``deltamic/render.py``) on the B200 kernels.

Same names, arguments and results as the reference:

* ``Fourier3dMesh(box_size, box_shape, device, dtype, OTF, narrowband_thresh)``
  (render.py:112-172) -- ``forward(Verts, Faces, Faces_coeff)`` returns the dense
  complex spectrum, zero outside the narrow band ``OTF > narrowband_thresh``
  (cuda_class.py:22); gradients flow to Verts and Faces_coeff;
* ``render_image_from_ftmesh`` (render.py:177-180), ``normalize_tensor``
  (render.py:5-6), ``compute_box_size`` (render.py:9-18),
  ``compute_spatial_frequency_grid`` (render.py:321-340), ``center_verts_in_box``
  (render.py:343-355).

Differences, all deliberate: the module runs on CUDA only (``device='cpu'``
raises -- there is no CPU fallback); the kernels compute in float32 (with the
fixed-point phases their error against a float64 evaluation is ~1e-6), so a
``dtype=torch.float64`` module casts its inputs to float32 and returns a
complex128 spectrum whose gradients flow back to the float64 inputs; the box
used for the phases is kept in float64.
"""
from __future__ import annotations

import numpy as np
import torch
from torch import nn

from . import ops

__all__ = ["Fourier3dMesh", "render_image_from_ftmesh", "normalize_tensor",
           "compute_box_size", "compute_spatial_frequency_grid", "center_verts_in_box"]


def normalize_tensor(t, contrast_variable=0):
    """Min-max normalisation ``((t - min)/(max - min) + c)/(1 + c)``."""
    lo, hi = t.min(), t.max()
    return ((t - lo) / (hi - lo) + contrast_variable) / (1 + contrast_variable)


def compute_box_size(verts, offset=0.1):
    """Cubic box around ``verts`` ([nv,3] numpy) with ``offset`` relative margin."""
    v = np.asarray(verts, dtype=np.float64)
    vmax, vmin = v.max(axis=0), v.min(axis=0)
    ext = vmax - vmin
    hi = vmax + ext * offset / 2
    lo = vmin - ext * offset / 2
    box = np.empty((3, 2))
    box[:, 0] = lo.min()
    box[:, 1] = hi.max()
    return box


def compute_spatial_frequency_grid(box_shape, box_size, device="cpu", dtype=torch.float):
    """Centred axes for box *lengths* ``box_size[3]`` (render.py:321-340)."""
    axes = []
    for d in range(3):
        n = int(box_shape[d])
        k = torch.arange(n, dtype=dtype, device=device)
        axes.append((2 * k - (n - 1)) * (np.pi / box_size[d]))
    return tuple(axes)


def center_verts_in_box(verts, box_size, offset=0.4):
    """Scale and translate ``verts`` (numpy, in place) into ``box_size``."""
    box = np.array(box_size)
    ext_v = verts.max(axis=0) - verts.min(axis=0)
    ext_b = box[:, 1] - box[:, 0]
    verts *= min(ext_b / ext_v)
    verts *= 1 - offset
    ext_v = verts.max(axis=0) - verts.min(axis=0)
    disp = 0.5 * (ext_b - ext_v)
    verts += box[:, 1] - verts.max(axis=0) - disp
    return verts


def render_image_from_ftmesh(ftmesh, OTF, box_shape):
    """``|ifftn(ftmesh * OTF)|`` over ``box_shape`` (cuFFT through torch.fft)."""
    return torch.abs(torch.fft.ifftn(ftmesh * OTF, list(box_shape)))


def _is_cuda(device) -> bool:
    try:
        return torch.device(device).type == "cuda"
    except (TypeError, RuntimeError):
        return False


class Fourier3dMesh(nn.Module):
    """meshFT layer: triangle mesh -> dense complex spectrum on the narrow band."""

    def __init__(self, box_size, box_shape, device="cpu", dtype=torch.float, OTF=None,
                 narrowband_thresh=0.01):
        super().__init__()
        if not _is_cuda(device):
            raise RuntimeError("deltamic_b200.Fourier3dMesh runs on CUDA devices only "
                               f"(got device={device!r}); there is no CPU path")
        if dtype not in (torch.float32, torch.float64):
            raise TypeError(f"Fourier3dMesh supports float32 and float64, not {dtype}")
        bs = torch.as_tensor(box_size).detach().cpu()
        self.grid = ops.FreqGrid(bs.double().numpy(), box_shape)
        self.box_size = torch.tensor(bs.numpy(), device=device, dtype=dtype)
        self.box_shape = list(box_shape)
        self.dtype = dtype
        self.device = device
        self.xi0, self.xi1, self.xi2 = self._compute_spatial_frequency_grid()
        if OTF is None:
            self.OTF = torch.ones(self.box_shape, device=device, dtype=dtype)
        else:
            self.OTF = OTF
        self.narrowband_thresh = narrowband_thresh
        self._band_key = None
        self._band = None

    def _compute_spatial_frequency_grid(self):
        out = []
        for d in range(3):
            n = self.box_shape[d]
            s = np.pi / (self.box_size[d, 1] - self.box_size[d, 0])
            k = torch.arange(n, dtype=self.dtype, device=self.device)
            out.append((2 * k - (n - 1)) * s)
        return tuple(out)

    def band(self) -> torch.Tensor:
        """Narrow-band voxel indices for the current ``OTF`` (recomputed when it changes)."""
        otf = self.OTF
        thr = float(self.narrowband_thresh)
        key = (otf.data_ptr(), otf._version, tuple(otf.shape), thr)
        if key != self._band_key or self._band is None:
            if tuple(otf.shape) != tuple(self.box_shape):
                raise ValueError("OTF must have shape box_shape")
            self._band = ops.narrowband(otf.detach().float().contiguous(), thr)
            self._band_key = key
        return self._band

    def forward(self, Verts, Faces, Faces_coeff):
        if self.dtype == torch.float64:
            ft = ops.meshft(Verts.float(), Faces, Faces_coeff.float(), self.grid, self.band())
            return ft.to(torch.complex128)
        return ops.meshft(Verts, Faces, Faces_coeff, self.grid, self.band())
