"""Drop-in rendering API of deltaMic (``deltamic/render.py``) on the B200 kernels.

Same names, arguments and results as the reference:

* ``Fourier3dMesh(box_size, box_shape, device, dtype, OTF, narrowband_thresh)``
  (render.py:112-172) -- ``forward(Verts, Faces, Faces_coeff)`` returns the dense
  complex spectrum, zero outside the narrow band ``OTF > narrowband_thresh``
  (cuda_class.py:22); gradients flow to Verts and Faces_coeff;
* ``render_image_from_ftmesh`` (render.py:177-180), ``normalize_tensor``
  (render.py:5-6), ``compute_box_size`` (render.py:9-18),
  ``compute_spatial_frequency_grid`` (render.py:321-340), ``center_verts_in_box``
  (render.py:343-355);
* ``fourier_from_mesh_narrowband_autofluorescence`` (render.py:228-318): surface
  plus enclosed-volume transform on the kernels of volume.cu, gradients for
  Verts and regint; its helpers ``get_internal_triangle_and_mesh_areas``,
  ``get_internal_triangle_and_mesh_areas_and_normals`` and
  ``compute_volume_manifold`` (render.py:184-226) are plain torch as in the
  reference.

Differences, all deliberate: the module runs on CUDA only (``device='cpu'``
raises -- there is no CPU fallback).  ``dtype=torch.float32`` runs the float32
kernels (fixed-point phases; error against a float64 evaluation ~1e-6);
``dtype=torch.float64`` runs the float64 kernels (the double arithmetic of the
reference's CPU path, Seps = sqrt(1.19209e-07), band selected on the float64 OTF)
and returns complex128.  ``render_image_from_ftmesh`` of a float32 spectrum that
``Fourier3dMesh`` returned (unmodified) runs the band-box DFTs of bandbox.cu,
which touch only the band's bounding box, for boxes of 64^3 voxels or more; other
spectra take ``abs(ifftn(ftmesh * OTF))`` on cuFFT.  ``normalize_tensor`` of a CUDA float32 /
float64 tensor runs the kernels of normalize.cu.  In the autofluorescence transform the
reference's value at xi = 0 (grids with every axis odd) is 0/0 = NaN; here it is
the limit of its volume term, ``1 - regint`` in all.
"""
from __future__ import annotations

import numpy as np
import torch
from torch import nn

from . import ops

__all__ = ["Fourier3dMesh", "render_image_from_ftmesh", "normalize_tensor",
           "compute_box_size", "compute_spatial_frequency_grid", "center_verts_in_box",
           "get_internal_triangle_and_mesh_areas",
           "get_internal_triangle_and_mesh_areas_and_normals", "compute_volume_manifold",
           "fourier_from_mesh_narrowband_autofluorescence"]


def normalize_tensor(t, contrast_variable=0):
    """Min-max normalisation ``((t - min)/(max - min) + c)/(1 + c)`` (render.py:5-6).

    A non-empty float32 / float64 CUDA tensor with a constant ``c`` runs the
    device kernels (two launches forward, two backward; gradient to ``t``).  A
    ``c`` that requires grad, or a host tensor, takes the eager expression."""
    c = contrast_variable
    if (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype in (torch.float32, torch.float64)
            and t.numel() > 0 and not (isinstance(c, torch.Tensor) and c.requires_grad)):
        return ops.normalize(t, float(c))
    lo, hi = t.min(), t.max()
    return ((t - lo) / (hi - lo) + c) / (1 + c)


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


_BB_PLANS: dict = {}


def _bandbox_plan(grid, band):
    """Cached (band-box plan, int64 band) of ``band`` on ``grid``: one host sync per
    new band.  The entry holds the band tensor itself, so its memory cannot be
    reused by another band while the entry lives."""
    key = (tuple(grid.box_size.ravel().tolist()), grid.shape, id(band), band._version)
    hit = _BB_PLANS.get(key)
    if hit is not None and hit[0] is band:
        return hit[1], hit[2]
    if len(_BB_PLANS) >= 8:
        _BB_PLANS.pop(next(iter(_BB_PLANS)))
    plan = ops.BandBox(grid, band)
    band64 = band.long()
    _BB_PLANS[key] = (band, plan, band64)
    return plan, band64


class _BandImage(torch.autograd.Function):
    """``|ifftn(ftmesh * OTF)|`` of a spectrum that is zero outside ``band``, by the
    band-box DFTs; backward gives the dense dL/dftmesh (zero off the band) and,
    for a real OTF, dL/dOTF = Re(conj(ftmesh) dL/dS)."""

    @staticmethod
    def forward(ctx, ftmesh, OTF, band, plan, band64):
        ft = ftmesh.reshape(-1).index_select(0, band64)
        otf = OTF.contiguous()
        img = ops.render_bandbox_image(ft, band, plan, otf)
        ctx.save_for_backward(ft, otf, band, band64)
        ctx.plan = plan
        ctx.shape = tuple(ftmesh.shape)
        return img

    @staticmethod
    def backward(ctx, g):
        ft, otf, band, band64 = ctx.saved_tensors
        plan = ctx.plan
        G = ops.render_bandbox_adjoint(ft, band, plan, otf, g.contiguous().float())
        gS = G * (1.0 / plan.grid.numel)  # dL/dS on the band
        g_ft = g_otf = None
        if ctx.needs_input_grad[0]:
            g_ft = torch.zeros(ctx.shape, dtype=torch.complex64, device=ft.device)
            g_ft.view(-1).index_copy_(0, band64, gS * otf.view(-1).index_select(0, band64))
        if ctx.needs_input_grad[1]:
            g_otf = torch.zeros(ctx.shape, dtype=torch.float32, device=ft.device)
            g_otf.view(-1).index_copy_(0, band64, (gS * ft.conj()).real)
        return g_ft, g_otf, None, None, None


# Below this many voxels the two cuFFT transforms of the dense route cost less than
# the band-box route's launches (and its backward recomputes z).
_BAND_ROUTE_MIN_VOXELS = 1 << 18


def _band_route(ftmesh, OTF, box_shape):
    info = getattr(ftmesh, "_dm_band", None)
    if info is None or info[2] != ftmesh._version or ftmesh.dtype != torch.complex64:
        return None
    if ftmesh.numel() < _BAND_ROUTE_MIN_VOXELS:
        return None
    if not (isinstance(OTF, torch.Tensor) and OTF.is_cuda and OTF.dtype == torch.float32
            and OTF.device == ftmesh.device and tuple(OTF.shape) == tuple(ftmesh.shape)):
        return None
    try:
        if [int(b) for b in box_shape] != list(ftmesh.shape):
            return None
    except (TypeError, ValueError):
        return None
    band, grid = info[0], info[1]
    if band.numel() == 0:
        return None
    plan, band64 = _bandbox_plan(grid, band)
    return (band, plan, band64) if plan.supported else None


def render_image_from_ftmesh(ftmesh, OTF, box_shape):
    """``|ifftn(ftmesh * OTF)|`` over ``box_shape`` (render.py:177-180).

    For a float32 spectrum straight from :class:`Fourier3dMesh` (zero off its
    narrow band; no in-place change since) with a real float32 OTF of the same
    shape and at least 64^3 voxels, the image comes from the band-box DFTs;
    otherwise from cuFFT."""
    route = _band_route(ftmesh, OTF, box_shape)
    if route is not None:
        band, plan, band64 = route
        return _BandImage.apply(ftmesh, OTF, band, plan, band64)
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
            o = otf.detach()
            o = o.double() if self.dtype == torch.float64 else o.float()
            self._band = ops.narrowband(o.contiguous(), thr)
            self._band_key = key
        return self._band

    def forward(self, Verts, Faces, Faces_coeff):
        if self.dtype == torch.float64:
            return ops.meshft64(Verts.double(), Faces, Faces_coeff.double(), self.grid,
                                self.band())
        band = self.band()
        out = ops.meshft(Verts, Faces, Faces_coeff, self.grid, band)
        out._dm_band = (band, self.grid, out._version)  # zero off this band
        return out


# ---------------------------------------------------------------------------
# Surface + enclosed-volume ("autofluorescence") transform

def _heron(Verts, Faces):
    pos = Verts[Faces]
    ls = torch.norm(pos - pos[:, [2, 0, 1]], dim=2)
    hp = ls.sum(dim=1) / 2
    return pos, (hp * (hp - ls[:, 0]) * (hp - ls[:, 1]) * (hp - ls[:, 2])) ** 0.5


def get_internal_triangle_and_mesh_areas_with_coeff(Verts, Faces, Faces_coeff):
    """Heron areas times the face coefficients and their sum (render.py:21-33)."""
    _, a = _heron(Verts, Faces)
    trisar = Faces_coeff * a
    return trisar, torch.sum(trisar)


def get_internal_triangle_and_mesh_areas(Verts, Faces):
    """Heron areas of the faces and their sum (render.py:184-199)."""
    _, trisar = _heron(Verts, Faces)
    return trisar, trisar.sum()


def get_internal_triangle_and_mesh_areas_and_normals(Verts, Faces):
    """Heron areas, their sum and the unnormalised normals
    ``p0 x p1 + p1 x p2 + p2 x p0`` (render.py:202-218)."""
    pos, trisar = _heron(Verts, Faces)
    nor = (torch.cross(pos[:, 0], pos[:, 1], dim=1) + torch.cross(pos[:, 1], pos[:, 2], dim=1)
           + torch.cross(pos[:, 2], pos[:, 0], dim=1))
    return trisar, trisar.sum(), nor


def compute_volume_manifold(Verts, Faces):
    """``-sum p0 . (p1 x p2) / 6`` (render.py:221-226)."""
    c = Verts[Faces]
    return -torch.sum(torch.sum(torch.cross(c[:, 1], c[:, 2], dim=1) * c[:, 0], dim=1)) / 6


def _axis_length(x: torch.Tensor) -> float:
    """Box length L of a centred axis ``(2k - (n-1)) pi / L`` (render.py:321-340)."""
    v = x.detach().double().cpu().numpy().reshape(-1)
    n = v.size
    if n == 0:
        raise ValueError("empty frequency axis")
    if n == 1:
        if v[0] != 0.0:
            raise ValueError("a one-point frequency axis must be [0]")
        return 1.0
    s = (v[-1] - v[0]) / (2 * (n - 1))
    k = 2 * np.arange(n) - (n - 1)
    if not s > 0 or np.max(np.abs(v - k * s)) > 1e-5 * np.max(np.abs(v)):
        raise ValueError("frequency axes must be centred grids (2k - (n-1)) pi / L, as "
                         "compute_spatial_frequency_grid makes them")
    return float(np.pi / s)


_AUTO_BANDS: dict = {}


def fourier_from_mesh_narrowband_autofluorescence(OTF, narrowband_thresh, regint, xi0, xi1,
                                                  xi2, Verts, Faces):
    """Dense surface + enclosed-volume spectrum (render.py:228-318): zero outside
    ``OTF > narrowband_thresh``, and on the band
    ``sum_k F_k (2 A_k / sum A + i (regint / regvol) xi . nor_k / |xi|^2)``.

    Vertex coordinates enter as given.  Gradients flow to ``Verts`` and to
    ``regint`` when it is a tensor.  The transform runs on the float32 kernels
    only: a float64 ``Verts`` raises ``TypeError`` (no silent change of
    precision)."""
    shape = (int(xi0.numel()), int(xi1.numel()), int(xi2.numel()))
    if tuple(OTF.shape) != shape:
        raise ValueError(f"OTF shape {tuple(OTF.shape)} does not match the axes {shape}")
    L = [_axis_length(x) for x in (xi0, xi1, xi2)]
    grid = ops.FreqGrid(np.array([[0.0, L[0]], [0.0, L[1]], [0.0, L[2]]]), shape)
    thr = float(narrowband_thresh)
    key = (OTF.data_ptr(), OTF._version, shape, thr)
    hit = _AUTO_BANDS.get(id(OTF))
    if hit is not None and hit[0] == key:
        band = hit[1]
    else:
        band = ops.narrowband(OTF.detach().float().contiguous(), thr)
        _AUTO_BANDS.clear()
        _AUTO_BANDS[id(OTF)] = (key, band)
    if Verts.dtype != torch.float32:
        raise TypeError("fourier_from_mesh_narrowband_autofluorescence runs in float32 "
                        f"(got Verts of {Verts.dtype})")
    return ops.volume_ft(Verts, Faces, regint, grid, band)
