"""Autograd operators over the C ABI: narrow band, meshFT, Gaussian OTF, image loss.

Every operator here launches the kernels of ``libdeltamic_b200.so`` on the current
CUDA stream; none has a CPU or PyTorch fallback.
"""
from __future__ import annotations

import ctypes
import weakref

import numpy as np
import torch

from . import _native as N

__all__ = ["FreqGrid", "narrowband", "band_is_hermitian", "band_eval_count", "band_box",
           "topology", "meshft", "meshft_list", "meshft64", "meshft64_list",
           "meshft64_backward_list", "meshft_xi", "meshft_xi_list", "meshft_xi_backward_list",
           "meshft_backward_list", "volume_list", "volume_backward_list", "volume_ft",
           "gaussian_otf", "image_loss", "adam_step"]


class FreqGrid:
    """Box and shape of a centred frequency grid (render.py:153-172).

    ``box_size`` is a [3,2] array-like (lower, upper corner per axis); it is kept
    in float64 for the kernels' phase arithmetic.
    """

    def __init__(self, box_size, box_shape):
        b = np.asarray(torch.as_tensor(box_size).detach().cpu().double().numpy(), np.float64)
        if b.shape != (3, 2):
            raise ValueError("box_size must have shape [3, 2]")
        self.box_size = b
        self.shape = tuple(int(s) for s in box_shape)
        if len(self.shape) != 3 or min(self.shape) <= 0:
            raise ValueError("box_shape must be 3 positive integers")
        self.numel = int(np.prod(self.shape))
        self.cbox = N.make_box(b, self.shape)

    def axes(self, dtype=torch.float32, device="cuda"):
        """xi0, xi1, xi2 as Fourier3dMesh computes them (in ``dtype``)."""
        bs = torch.tensor(self.box_size, dtype=dtype, device=device)
        out = []
        for d in range(3):
            n = self.shape[d]
            s = np.pi / (bs[d, 1] - bs[d, 0])
            k = torch.arange(n, dtype=dtype, device=device)
            out.append((2 * k - (n - 1)) * s)
        return tuple(out)


# ---------------------------------------------------------------------------
# narrow band

def narrowband(otf: torch.Tensor, thresh: float) -> torch.Tensor:
    """Flat C-order indices (int32) of ``otf > thresh``, compared in the OTF's own
    precision (float32 or float64); synchronises to learn the count."""
    otf = otf.detach()
    N.require_cuda(otf, "OTF")
    if otf.dtype not in (torch.float32, torch.float64):
        raise TypeError(f"OTF must be float32 or float64, not {otf.dtype}")
    otf = otf.contiguous()
    n = otf.numel()
    lib = N.lib()
    idx = torch.empty(max(n, 1), dtype=torch.int32, device=otf.device)
    cnt = torch.zeros(1, dtype=torch.int64, device=otf.device)
    ws = N.WORKSPACES.get("band", lib.dm_narrowband_workspace_size(n), otf.device)
    if otf.dtype == torch.float64:
        N.check(lib.dm_narrowband_compact64(N.ptr(otf), n, float(thresh), N.ptr(idx),
                                            N.ptr(cnt), N.ptr(ws), ws.numel(),
                                            N.stream_ptr(otf.device)), "dm_narrowband_compact64")
    else:
        N.check(lib.dm_narrowband_compact(N.ptr(otf), n, float(thresh), N.ptr(idx), N.ptr(cnt),
                                          N.ptr(ws), ws.numel(), N.stream_ptr(otf.device)),
                "dm_narrowband_compact")
    c = int(cnt.item())
    band = idx[:c].clone()
    flag = torch.zeros(1, dtype=torch.int32, device=otf.device)
    N.check(lib.dm_narrowband_hermitian(N.ptr(band), c, n, N.ptr(flag),
                                        N.stream_ptr(otf.device)), "dm_narrowband_hermitian")
    _HERM[id(band)] = (weakref.ref(band), bool(flag.item()))
    return band


# Bands from narrowband() that are closed under xi -> -xi (the meshFT calls then
# evaluate half of them); keyed by id with a weak reference to the tensor.
_HERM: dict = {}


def band_is_hermitian(band: torch.Tensor) -> bool:
    """True for a band made by narrowband() whose voxel set is symmetric about the
    grid centre (every Gaussian OTF gives one)."""
    e = _HERM.get(id(band))
    if e is None or e[0]() is not band:
        return False
    return e[1]


def band_eval_count(band: torch.Tensor) -> int:
    """Frequencies the meshFT kernels evaluate for ``band``: half (rounded up)
    of a mirror-symmetric band, else all of it."""
    n = int(band.numel())
    return (n + 1) // 2 if band_is_hermitian(band) else n


def band_box(grid: FreqGrid, band) -> N.DmBox:
    """The C box of ``grid`` with the DM_BAND_* flags of ``band`` (a tensor from
    narrowband(), or a bool: the band is known to be mirror-symmetric)."""
    herm = band if isinstance(band, bool) else band_is_hermitian(band)
    b = N.DmBox.from_buffer_copy(grid.cbox)
    b.band_flags = N.DM_BAND_HERMITIAN if herm else 0
    return b


def order_band_by_radius(band: torch.Tensor, grid: FreqGrid) -> torch.Tensor:
    """The band's voxel indices sorted by |xi| (stable).  The meshFT calls accept
    the band in any order; neighbouring threads then see similar frequencies and
    take the same evaluation path more often."""
    if band.numel() == 0:
        return band
    n0, n1, n2 = grid.shape
    idx = band.long()
    k0 = idx // (n1 * n2)
    k1 = (idx // n2) % n1
    k2 = idx % n2
    L = grid.box_size[:, 1] - grid.box_size[:, 0]
    r2 = (((2 * k0 - (n0 - 1)) / L[0]) ** 2 + ((2 * k1 - (n1 - 1)) / L[1]) ** 2
          + ((2 * k2 - (n2 - 1)) / L[2]) ** 2)
    order = torch.sort(r2, stable=True).indices
    return band[order].contiguous()


# ---------------------------------------------------------------------------
# topology cache (vertex <- face CSR), keyed by the faces tensor

_TOPO: dict = {}


def topology(faces: torch.Tensor, nv: int) -> torch.Tensor:
    """CSR incidence buffer for ``faces`` (built once; face indices validated).

    Cached per faces tensor (by identity, held weakly) and its version counter."""
    key = (faces._version, int(nv), faces.data_ptr(), tuple(faces.shape))
    hit = _TOPO.get(id(faces))
    if hit is not None and hit[0]() is faces and hit[1] == key:
        return hit[2]
    for k in [k for k, v in _TOPO.items() if v[0]() is None]:
        del _TOPO[k]
    lib = N.lib()
    nt = faces.shape[0]
    if nt:
        lo, hi = int(faces.min()), int(faces.max())
        if lo < 0 or hi >= nv:
            raise IndexError(f"face index out of range [0, {nv}): min {lo}, max {hi}")
    buf = torch.zeros(lib.dm_topology_size(nv, nt), dtype=torch.uint8, device=faces.device)
    N.check(lib.dm_topology_build(N.ptr(faces), nt, nv, N.ptr(buf), buf.numel(),
                                  N.stream_ptr(faces.device)), "dm_topology_build")
    _TOPO[id(faces)] = (weakref.ref(faces), key, buf)
    return buf


def _check_mesh(verts, faces, coeff):
    N.require_cuda(verts, "Verts", torch.float32)
    N.require_cuda(faces, "Faces", torch.int64)
    N.require_cuda(coeff, "Faces_coeff", torch.float32)
    if verts.dim() != 2 or verts.shape[1] != 3:
        raise ValueError("Verts must have shape [nv, 3]")
    if faces.dim() != 2 or faces.shape[1] != 3:
        raise ValueError("Faces must have shape [nt, 3]")
    if coeff.shape != (faces.shape[0],):
        raise ValueError("Faces_coeff must have shape [nt]")


def meshft_list(verts, faces, coeff, grid: FreqGrid, band, otf=None, spectrum=None):
    """Forward only: ft_list[n_band] (complex64); optionally scatter ft*otf into ``spectrum``."""
    lib = N.lib()
    nv, nt, nb = verts.shape[0], faces.shape[0], band.numel()
    ft = torch.empty(nb, dtype=torch.complex64, device=verts.device)
    ws = N.WORKSPACES.get("fwd", lib.dm_meshft_forward_workspace_size(nv, nt, nb), verts.device)
    N.check(lib.dm_meshft_forward(
        N.ptr(verts), nv, N.ptr(faces), nt, N.ptr(coeff), ctypes.byref(band_box(grid, band)),
        N.ptr(band), nb, N.ptr(otf), N.ptr(ft), N.ptr(spectrum), N.ptr(ws), ws.numel(),
        N.stream_ptr(verts.device)), "dm_meshft_forward")
    return ft


def meshft_backward_list(verts, faces, coeff, grid: FreqGrid, band, ft, grad_list=None,
                         grad_grid=None, otf=None, scale=1.0, want_coeff=True, want_otf=False):
    """Backward only: (grad_verts, grad_coeff | None, grad_otf_band | None)."""
    lib = N.lib()
    nv, nt, nb = verts.shape[0], faces.shape[0], band.numel()
    gv = torch.empty_like(verts)
    gc = torch.empty_like(coeff) if want_coeff else None
    go = torch.empty(nb, dtype=torch.float32, device=verts.device) if want_otf else None
    topo = topology(faces, nv)
    ws = N.WORKSPACES.get("bwd", lib.dm_meshft_backward_workspace_size(nv, nt, nb), verts.device)
    N.check(lib.dm_meshft_backward(
        N.ptr(verts), nv, N.ptr(faces), nt, N.ptr(coeff), ctypes.byref(band_box(grid, band)),
        N.ptr(band), nb, N.ptr(grad_list), N.ptr(grad_grid), N.ptr(otf), float(scale), N.ptr(ft), N.ptr(topo),
        N.ptr(gv), N.ptr(gc), N.ptr(go), N.ptr(ws), ws.numel(), N.stream_ptr(verts.device)),
        "dm_meshft_backward")
    return gv, gc, go


class _MeshFT(torch.autograd.Function):
    """Dense meshFT: complex64 grid, ft on the band and 0 elsewhere (cuda_class.py:16-41)."""

    @staticmethod
    def forward(ctx, verts, faces, coeff, grid, band):
        out = torch.zeros(grid.shape, dtype=torch.complex64, device=verts.device)
        ft = meshft_list(verts, faces, coeff, grid, band, spectrum=out)
        ctx.save_for_backward(verts, faces, coeff, band, ft)
        ctx.grid = grid
        return out

    @staticmethod
    def backward(ctx, g):
        verts, faces, coeff, band, ft = ctx.saved_tensors
        g = g.contiguous()
        if g.dtype != torch.complex64:
            g = g.to(torch.complex64)
        gv, gc, _ = meshft_backward_list(verts, faces, coeff, ctx.grid, band, ft, grad_grid=g,
                                         want_coeff=ctx.needs_input_grad[2])
        return gv, None, gc, None, None


def meshft(verts, faces, coeff, grid: FreqGrid, band) -> torch.Tensor:
    """Differentiable dense meshFT (gradients for verts and coeff)."""
    _check_mesh(verts, faces, coeff)
    return _MeshFT.apply(verts.contiguous(), faces.contiguous(), coeff.contiguous(), grid, band)


# ---------------------------------------------------------------------------
# float32 meshFT on an explicit frequency list (split phase; any frequencies)

def meshft_xi_list(verts, faces, coeff, xi_list):
    """ft_list[n] (complex64) of the mesh (vertex coordinates as given) at the rows
    of ``xi_list`` [n, 3] float32."""
    _check_mesh(verts, faces, coeff)
    N.require_cuda(xi_list, "xi_list", torch.float32)
    lib = N.lib()
    nv, nt, n = verts.shape[0], faces.shape[0], xi_list.shape[0]
    ft = torch.empty(n, dtype=torch.complex64, device=verts.device)
    ws = N.WORKSPACES.get("fwd_xi", lib.dm_meshft_forward_xi_workspace_size(nv, nt, n),
                          verts.device)
    N.check(lib.dm_meshft_forward_xi(N.ptr(verts), nv, N.ptr(faces), nt, N.ptr(coeff),
                                     N.ptr(xi_list.contiguous()), n, N.ptr(ft), N.ptr(ws),
                                     ws.numel(), N.stream_ptr(verts.device)),
            "dm_meshft_forward_xi")
    return ft


def meshft_xi_backward_list(verts, faces, coeff, xi_list, grad_list, ft, want_coeff=True):
    """(grad_verts, grad_coeff | None) of :func:`meshft_xi_list` for the cotangent
    ``grad_list`` (complex64 on the list)."""
    lib = N.lib()
    nv, nt, n = verts.shape[0], faces.shape[0], xi_list.shape[0]
    gv = torch.empty_like(verts)
    gc = torch.empty_like(coeff) if want_coeff else None
    topo = topology(faces, nv)
    ws = N.WORKSPACES.get("bwd_xi", lib.dm_meshft_backward_xi_workspace_size(nv, nt, n),
                          verts.device)
    N.check(lib.dm_meshft_backward_xi(
        N.ptr(verts), nv, N.ptr(faces), nt, N.ptr(coeff), N.ptr(grad_list.contiguous()),
        N.ptr(ft.contiguous()), N.ptr(xi_list.contiguous()), n, N.ptr(topo), N.ptr(gv),
        N.ptr(gc), N.ptr(ws), ws.numel(), N.stream_ptr(verts.device)), "dm_meshft_backward_xi")
    return gv, gc


class _MeshFTXi(torch.autograd.Function):
    """ft_list on an explicit frequency list (float32 or float64 by the inputs);
    gradients for verts and coeff."""

    @staticmethod
    def forward(ctx, verts, coeff, faces, xi_list):
        if verts.dtype == torch.float64:
            ft = meshft64_list(verts, faces, coeff, xi_list=xi_list)
        else:
            ft = meshft_xi_list(verts, faces, coeff, xi_list)
        ctx.save_for_backward(verts, coeff, faces, xi_list, ft)
        return ft

    @staticmethod
    def backward(ctx, g):
        verts, coeff, faces, xi_list, ft = ctx.saved_tensors
        g = g.contiguous().to(ft.dtype)
        want_c = ctx.needs_input_grad[1]
        if verts.dtype == torch.float64:
            gv, gc = meshft64_backward_list(verts, faces, coeff, ft, xi_list=xi_list,
                                            grad_list=g, want_coeff=want_c)
        else:
            gv, gc = meshft_xi_backward_list(verts, faces, coeff, xi_list, g, ft,
                                             want_coeff=want_c)
        return gv, gc, None, None


def meshft_xi(verts, faces, coeff, xi_list) -> torch.Tensor:
    """Differentiable ft_list at explicit frequencies (vertex coordinates as
    given): float32 inputs -> complex64 (split-phase kernels), float64 inputs ->
    complex128 (float64 kernels)."""
    if verts.dtype == torch.float64:
        _check_mesh64(verts, faces, coeff)
        N.require_cuda(xi_list, "xi_list", torch.float64)
    else:
        _check_mesh(verts, faces, coeff)
        N.require_cuda(xi_list, "xi_list", torch.float32)
    return _MeshFTXi.apply(verts.contiguous(), coeff.contiguous(), faces.contiguous(),
                           xi_list.contiguous())


# ---------------------------------------------------------------------------
# float64 meshFT (the reference's double dispatch, fourier3d_cuda_kernel.cu:238-416)

def _check_mesh64(verts, faces, coeff):
    N.require_cuda(verts, "Verts", torch.float64)
    N.require_cuda(faces, "Faces", torch.int64)
    N.require_cuda(coeff, "Faces_coeff", torch.float64)
    if verts.dim() != 2 or verts.shape[1] != 3:
        raise ValueError("Verts must have shape [nv, 3]")
    if faces.dim() != 2 or faces.shape[1] != 3:
        raise ValueError("Faces must have shape [nt, 3]")
    if coeff.shape != (faces.shape[0],):
        raise ValueError("Faces_coeff must have shape [nt]")


def meshft64_list(verts, faces, coeff, grid: FreqGrid = None, band=None, xi_list=None,
                  otf=None, spectrum=None):
    """Float64 forward: ft_list (complex128) on a grid band (``grid`` + ``band``) or
    on an explicit ``xi_list`` [n, 3] float64 (vertex coordinates as given);
    optionally scatters ft*otf into the complex128 ``spectrum`` (grid band only)."""
    lib = N.lib()
    nv, nt = verts.shape[0], faces.shape[0]
    n = band.numel() if band is not None else xi_list.shape[0]
    ft = torch.empty(n, dtype=torch.complex128, device=verts.device)
    ws = N.WORKSPACES.get("fwd64", lib.dm_meshft64_forward_workspace_size(nv, nt, n),
                          verts.device)
    box = ctypes.byref(grid.cbox) if band is not None else None
    N.check(lib.dm_meshft64_forward(
        N.ptr(verts), nv, N.ptr(faces), nt, N.ptr(coeff), box, N.ptr(band), N.ptr(xi_list), n,
        N.ptr(otf), N.ptr(ft), N.ptr(spectrum), N.ptr(ws), ws.numel(),
        N.stream_ptr(verts.device)), "dm_meshft64_forward")
    return ft


def meshft64_backward_list(verts, faces, coeff, ft, grid: FreqGrid = None, band=None,
                           xi_list=None, grad_list=None, grad_grid=None, otf=None, scale=1.0,
                           want_coeff=True):
    """Float64 backward: (grad_verts, grad_coeff | None) for the cotangent of
    :func:`meshft64_list`'s result (``grad_list`` complex128 on the frequencies, or
    ``grad_grid`` on the grid band)."""
    lib = N.lib()
    nv, nt = verts.shape[0], faces.shape[0]
    n = band.numel() if band is not None else xi_list.shape[0]
    gv = torch.empty_like(verts)
    gc = torch.empty_like(coeff) if want_coeff else None
    topo = topology(faces, nv)
    ws = N.WORKSPACES.get("bwd64", lib.dm_meshft64_backward_workspace_size(nv, nt, n),
                          verts.device)
    box = ctypes.byref(grid.cbox) if band is not None else None
    N.check(lib.dm_meshft64_backward(
        N.ptr(verts), nv, N.ptr(faces), nt, N.ptr(coeff), box, N.ptr(band), N.ptr(xi_list), n,
        N.ptr(grad_list), N.ptr(grad_grid), N.ptr(otf), float(scale), N.ptr(ft), N.ptr(topo),
        N.ptr(gv), N.ptr(gc), N.ptr(ws), ws.numel(), N.stream_ptr(verts.device)),
        "dm_meshft64_backward")
    return gv, gc


class _MeshFT64(torch.autograd.Function):
    """Dense float64 meshFT: complex128 grid, ft on the band and 0 elsewhere."""

    @staticmethod
    def forward(ctx, verts, faces, coeff, grid, band):
        out = torch.zeros(grid.shape, dtype=torch.complex128, device=verts.device)
        ft = meshft64_list(verts, faces, coeff, grid, band, spectrum=out)
        ctx.save_for_backward(verts, faces, coeff, band, ft)
        ctx.grid = grid
        return out

    @staticmethod
    def backward(ctx, g):
        verts, faces, coeff, band, ft = ctx.saved_tensors
        g = g.contiguous()
        if g.dtype != torch.complex128:
            g = g.to(torch.complex128)
        gv, gc = meshft64_backward_list(verts, faces, coeff, ft, ctx.grid, band, grad_grid=g,
                                        want_coeff=ctx.needs_input_grad[2])
        return gv, None, gc, None, None


def meshft64(verts, faces, coeff, grid: FreqGrid, band) -> torch.Tensor:
    """Differentiable dense float64 meshFT (gradients for verts and coeff)."""
    _check_mesh64(verts, faces, coeff)
    return _MeshFT64.apply(verts.contiguous(), faces.contiguous(), coeff.contiguous(), grid,
                           band)


# ---------------------------------------------------------------------------
# surface + enclosed-volume transform (render.py:228-318)

def volume_list(verts, faces, regint, grid: FreqGrid, band, otf=None, spectrum=None):
    """Forward of the surface + enclosed-volume transform: ``(ft_list, vol_list)``
    (complex64 on the band); optionally scatters ft*otf into ``spectrum``.
    ``regint`` is a one-element float32 CUDA tensor; ``grid`` has lower corner 0."""
    lib = N.lib()
    nv, nt, nb = verts.shape[0], faces.shape[0], band.numel()
    ft = torch.empty(nb, dtype=torch.complex64, device=verts.device)
    vol = torch.empty(nb, dtype=torch.complex64, device=verts.device)
    ws = N.WORKSPACES.get("vol_fwd", lib.dm_meshft_volume_forward_workspace_size(nv, nt, nb),
                          verts.device)
    N.check(lib.dm_meshft_volume_forward(
        N.ptr(verts), nv, N.ptr(faces), nt, N.ptr(regint), ctypes.byref(band_box(grid, band)),
        N.ptr(band), nb, N.ptr(otf), N.ptr(ft), N.ptr(vol), N.ptr(spectrum), N.ptr(ws),
        ws.numel(), N.stream_ptr(verts.device)), "dm_meshft_volume_forward")
    return ft, vol


def volume_backward_list(verts, faces, regint, grid: FreqGrid, band, ft, vol, grad_list=None,
                         grad_grid=None, otf=None, scale=1.0, want_regint=True):
    """Backward of :func:`volume_list`: ``(grad_verts, grad_regint[1] | None)``."""
    lib = N.lib()
    nv, nt, nb = verts.shape[0], faces.shape[0], band.numel()
    gv = torch.empty_like(verts)
    gr = torch.empty(1, dtype=torch.float32, device=verts.device) if want_regint else None
    topo = topology(faces, nv)
    ws = N.WORKSPACES.get("vol_bwd", lib.dm_meshft_volume_backward_workspace_size(nv, nt, nb),
                          verts.device)
    N.check(lib.dm_meshft_volume_backward(
        N.ptr(verts), nv, N.ptr(faces), nt, N.ptr(regint), ctypes.byref(band_box(grid, band)),
        N.ptr(band), nb, N.ptr(grad_list), N.ptr(grad_grid), N.ptr(otf), float(scale),
        N.ptr(ft), N.ptr(vol), N.ptr(topo), N.ptr(gv), N.ptr(gr), N.ptr(ws), ws.numel(),
        N.stream_ptr(verts.device)), "dm_meshft_volume_backward")
    return gv, gr


class _VolumeFT(torch.autograd.Function):
    """Dense surface + enclosed-volume transform: complex64 grid, ft on the band and
    0 elsewhere (render.py:228-318); gradients for verts and regint."""

    @staticmethod
    def forward(ctx, verts, regint, faces, grid, band):
        out = torch.zeros(grid.shape, dtype=torch.complex64, device=verts.device)
        ft, vol = volume_list(verts, faces, regint, grid, band, spectrum=out)
        ctx.save_for_backward(verts, regint, faces, band, ft, vol)
        ctx.grid = grid
        return out

    @staticmethod
    def backward(ctx, g):
        verts, regint, faces, band, ft, vol = ctx.saved_tensors
        g = g.contiguous()
        if g.dtype != torch.complex64:
            g = g.to(torch.complex64)
        gv, gr = volume_backward_list(verts, faces, regint, ctx.grid, band, ft, vol, grad_grid=g,
                                      want_regint=ctx.needs_input_grad[1])
        return gv, gr, None, None, None


def volume_ft(verts, faces, regint, grid: FreqGrid, band) -> torch.Tensor:
    """Differentiable dense surface + enclosed-volume transform (gradients for
    ``verts`` and a tensor ``regint``).  ``grid`` must have lower corner 0: the
    vertex coordinates enter as given."""
    N.require_cuda(verts, "Verts", torch.float32)
    N.require_cuda(faces, "Faces", torch.int64)
    if verts.dim() != 2 or verts.shape[1] != 3:
        raise ValueError("Verts must have shape [nv, 3]")
    if faces.dim() != 2 or faces.shape[1] != 3:
        raise ValueError("Faces must have shape [nt, 3]")
    if np.any(grid.box_size[:, 0] != 0.0):
        raise ValueError("the volume transform takes vertex coordinates as given: "
                         "grid.box_size[:, 0] must be 0")
    r = regint if isinstance(regint, torch.Tensor) else torch.tensor(float(regint))
    if r.numel() != 1:
        raise ValueError("regint must be a scalar")
    r = r.to(device=verts.device, dtype=torch.float32).reshape(1)
    return _VolumeFT.apply(verts.contiguous(), r, faces.contiguous(), grid, band)


# ---------------------------------------------------------------------------
# Gaussian OTF

class _GaussianOTF(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sigma, x0, x1, x2):
        lib = N.lib()
        n = (x0.numel(), x1.numel(), x2.numel())
        otf = torch.empty(n, dtype=sigma.dtype, device=sigma.device)
        f = lib.dm_gaussian_otf64 if sigma.dtype == torch.float64 else lib.dm_gaussian_otf
        N.check(f(N.ptr(sigma), N.ptr(x0), n[0], N.ptr(x1), n[1], N.ptr(x2), n[2], N.ptr(otf),
                  N.stream_ptr(sigma.device)), "dm_gaussian_otf")
        ctx.save_for_backward(otf, x0, x1, x2)
        return otf

    @staticmethod
    def backward(ctx, g):
        otf, x0, x1, x2 = ctx.saved_tensors
        if not ctx.needs_input_grad[0]:
            return None, None, None, None
        return sigma_grad_dense(g.contiguous().to(otf.dtype), otf, x0, x1, x2), None, None, None


def sigma_grad_dense(gotf, otf, x0, x1, x2, band=None):
    """d loss/d sigma from an OTF gradient (dense, or on ``band`` indices); in the
    OTF's precision (float32 or float64)."""
    lib = N.lib()
    n = band.numel() if band is not None else otf.numel()
    gs = torch.empty(3, 3, dtype=otf.dtype, device=otf.device)
    ws = N.WORKSPACES.get("otfgrad", lib.dm_gaussian_otf_grad_workspace_size(n), otf.device)
    f = (lib.dm_gaussian_otf64_sigma_grad if otf.dtype == torch.float64
         else lib.dm_gaussian_otf_sigma_grad)
    N.check(f(N.ptr(gotf), N.ptr(band), n, N.ptr(otf), N.ptr(x0), x0.numel(), N.ptr(x1),
              x1.numel(), N.ptr(x2), x2.numel(), N.ptr(gs), N.ptr(ws), ws.numel(),
              N.stream_ptr(otf.device)), "dm_gaussian_otf_sigma_grad")
    return gs


def gaussian_otf(sigma, xi0, xi1, xi2) -> torch.Tensor:
    """exp(-(xi^T sigma xi)/2) on the grid of the axes, differentiable in sigma;
    float64 when sigma or the axes are float64 (the float64 kernel), else float32."""
    N.require_cuda(sigma, "sigma")
    f64 = sigma.dtype == torch.float64 or xi0.dtype == torch.float64
    rt = torch.float64 if f64 else torch.float32
    sigma = sigma.to(rt).contiguous()
    if sigma.shape != (3, 3):
        raise ValueError("sigma must be a 3x3 matrix")
    axes = []
    for name, x in (("xi0", xi0), ("xi1", xi1), ("xi2", xi2)):
        N.require_cuda(x, name)
        axes.append(x.detach().to(rt).contiguous())
    return _GaussianOTF.apply(sigma, *axes)


# ---------------------------------------------------------------------------
# fused image stage and Adam

LOSS_KINDS = {"sum": 0, "mse": 1}


def image_loss(z, kind="sum", target=None, contrast=0.0, want_grad=True, want_image=False):
    """(loss[1], image | None, dL/dz | None) for z = ifftn(ftmesh*OTF), complex64."""
    lib = N.lib()
    N.require_cuda(z, "z", torch.complex64)
    n = z.numel()
    k = LOSS_KINDS[kind]
    if k == 1:
        N.require_cuda(target, "target", torch.float32)
        if target.numel() != n:
            raise ValueError("target must have the image's shape")
    loss = torch.empty(1, dtype=torch.float32, device=z.device)
    img = torch.empty(z.shape, dtype=torch.float32, device=z.device) if want_image else None
    gz = torch.empty_like(z) if want_grad else None
    ws = N.WORKSPACES.get("img", lib.dm_image_loss_workspace_size(n), z.device)
    N.check(lib.dm_image_loss(N.ptr(z), n, k, N.ptr(target), float(contrast), N.ptr(img),
                              N.ptr(loss), N.ptr(gz), N.ptr(ws), ws.numel(),
                              N.stream_ptr(z.device)), "dm_image_loss")
    return loss, img, gz


def band_bounds(band: torch.Tensor, grid: FreqGrid) -> tuple:
    """(lo0, lo1, lo2, hi0, hi1, hi2): per-axis smallest and largest voxel index of
    the band (synchronises to read them)."""
    N.require_cuda(band, "band", torch.int32)
    out = torch.empty(6, dtype=torch.int32, device=band.device)
    N.check(N.lib().dm_band_bounds(N.ptr(band), band.numel(), ctypes.byref(grid.cbox),
                                   N.ptr(out), N.stream_ptr(band.device)), "dm_band_bounds")
    return tuple(int(v) for v in out.cpu().tolist())


class BandBox:
    """Plan of the band-box render of ``band`` on ``grid``: the band's bounding box
    (host copy) and whether the library serves it."""

    def __init__(self, grid: FreqGrid, band: torch.Tensor):
        self.grid = grid
        self.bounds_tuple = band_bounds(band, grid) if band.numel() else (0, 0, 0, -1, -1, -1)
        self.bounds = (ctypes.c_int32 * 6)(*self.bounds_tuple)
        self.box = band_box(grid, band)
        lib = N.lib()
        self.supported = band.numel() > 0 and bool(
            lib.dm_render_loss_bandbox_supported(ctypes.byref(self.box), self.bounds))
        self.ws_bytes = (int(lib.dm_render_loss_bandbox_workspace_size(ctypes.byref(self.box),
                                                                       self.bounds))
                         if self.supported else 0)

    @property
    def extent(self) -> tuple:
        b = self.bounds_tuple
        return tuple(b[3 + d] - b[d] + 1 for d in range(3))


def render_loss_bandbox(ft, band, plan: BandBox, otf, kind="sum", target=None, contrast=0.0,
                        want_grad=True, want_image=False):
    """(loss[1], image | None, G | None) for S = ft * otf on the band: the loss of
    normalize(|ifftn(S)|) as image_loss computes it, and G = fftn(dL/dz) on the band
    (the grad_list of meshft_backward_list with otf and scale = 1/numel)."""
    lib = N.lib()
    if not plan.supported:
        raise N.DeltaMicError(N.DM_ERR_UNSUPPORTED, "render_loss_bandbox")
    N.require_cuda(ft, "ft", torch.complex64)
    N.require_cuda(otf, "OTF", torch.float32)
    k = LOSS_KINDS[kind]
    n = plan.grid.numel
    if k == 1:
        N.require_cuda(target, "target", torch.float32)
        if target.numel() != n:
            raise ValueError("target must have the image's shape")
    dev = ft.device
    loss = torch.empty(1, dtype=torch.float32, device=dev)
    G = torch.empty_like(ft) if want_grad else None
    img = torch.empty(plan.grid.shape, dtype=torch.float32, device=dev) if want_image else None
    ws = N.WORKSPACES.get("bandbox", plan.ws_bytes, dev)
    N.check(lib.dm_render_loss_bandbox(
        N.ptr(ft), N.ptr(band), band.numel(), ctypes.byref(plan.box), plan.bounds, N.ptr(otf), k,
        N.ptr(target), float(contrast), N.ptr(loss), N.ptr(G), N.ptr(img), N.ptr(ws), ws.numel(),
        N.stream_ptr(dev)), "dm_render_loss_bandbox")
    return loss, img, G


def render_bandbox_image(ft, band, plan: BandBox, otf):
    """|ifftn(S)| over the box for S = ft * otf on the band and 0 elsewhere
    (render_image_from_ftmesh of a band-limited spectrum), by the band-box DFTs."""
    lib = N.lib()
    if not plan.supported:
        raise N.DeltaMicError(N.DM_ERR_UNSUPPORTED, "render_bandbox_image")
    N.require_cuda(ft, "ft", torch.complex64)
    N.require_cuda(otf, "OTF", torch.float32)
    dev = ft.device
    loss = torch.empty(1, dtype=torch.float32, device=dev)
    img = torch.empty(plan.grid.shape, dtype=torch.float32, device=dev)
    ws = N.WORKSPACES.get("bandbox", plan.ws_bytes, dev)
    N.check(lib.dm_render_loss_bandbox(
        N.ptr(ft), N.ptr(band), band.numel(), ctypes.byref(plan.box), plan.bounds, N.ptr(otf), 2,
        None, 0.0, N.ptr(loss), None, N.ptr(img), N.ptr(ws), ws.numel(), N.stream_ptr(dev)),
        "dm_render_loss_bandbox")
    return img


def render_bandbox_adjoint(ft, band, plan: BandBox, otf, grad_image):
    """G = fftn(dL/dz) on the band for the cotangent ``grad_image`` = dL/d|z| of
    :func:`render_bandbox_image`; dL/dS on the band is G / numel."""
    lib = N.lib()
    if not plan.supported:
        raise N.DeltaMicError(N.DM_ERR_UNSUPPORTED, "render_bandbox_adjoint")
    N.require_cuda(ft, "ft", torch.complex64)
    N.require_cuda(otf, "OTF", torch.float32)
    N.require_cuda(grad_image, "grad_image", torch.float32)
    if grad_image.numel() != plan.grid.numel:
        raise ValueError("grad_image must have the image's shape")
    dev = ft.device
    loss = torch.empty(1, dtype=torch.float32, device=dev)
    G = torch.empty_like(ft)
    ws = N.WORKSPACES.get("bandbox", plan.ws_bytes, dev)
    N.check(lib.dm_render_loss_bandbox(
        N.ptr(ft), N.ptr(band), band.numel(), ctypes.byref(plan.box), plan.bounds, N.ptr(otf), 2,
        N.ptr(grad_image), 0.0, N.ptr(loss), N.ptr(G), None, N.ptr(ws), ws.numel(),
        N.stream_ptr(dev)), "dm_render_loss_bandbox")
    return G


# ---------------------------------------------------------------------------
# normalize_tensor (render.py:5-6)

def normalize_stats(t, contrast=0.0, want_out=True):
    """(out | None, stats[2] = (min, max)) of normalize_tensor for a contiguous
    float32 / float64 CUDA tensor ``t``."""
    if t.dtype not in (torch.float32, torch.float64):
        raise TypeError(f"normalize runs on float32 / float64 tensors, not {t.dtype}")
    N.require_cuda(t, "t", t.dtype)
    if t.numel() == 0:
        raise RuntimeError("normalize_tensor of an empty tensor (min() has no value)")
    lib = N.lib()
    f = lib.dm_normalize64 if t.dtype == torch.float64 else lib.dm_normalize
    stats = torch.empty(2, dtype=t.dtype, device=t.device)
    out = torch.empty_like(t) if want_out else None
    ws = N.WORKSPACES.get("normalize", lib.dm_normalize_workspace_size(t.numel()), t.device)
    N.check(f(N.ptr(t), t.numel(), float(contrast), N.ptr(out), N.ptr(stats), N.ptr(ws),
              ws.numel(), N.stream_ptr(t.device)), "dm_normalize")
    return out, stats


def normalize_backward(t, grad_out, stats, contrast=0.0):
    """dL/dt of normalize_tensor for the cotangent ``grad_out``."""
    lib = N.lib()
    f = lib.dm_normalize64_backward if t.dtype == torch.float64 else lib.dm_normalize_backward
    g = grad_out.contiguous()
    if g.dtype != t.dtype:
        g = g.to(t.dtype)
    out = torch.empty_like(t)
    ws = N.WORKSPACES.get("normalize", lib.dm_normalize_workspace_size(t.numel()), t.device)
    N.check(f(N.ptr(t), N.ptr(g), t.numel(), float(contrast), N.ptr(stats), N.ptr(out),
              N.ptr(ws), ws.numel(), N.stream_ptr(t.device)), "dm_normalize_backward")
    return out


class _Normalize(torch.autograd.Function):
    @staticmethod
    def forward(ctx, t, contrast):
        out, stats = normalize_stats(t, contrast)
        ctx.save_for_backward(t, stats)
        ctx.contrast = contrast
        return out

    @staticmethod
    def backward(ctx, g):
        t, stats = ctx.saved_tensors
        return normalize_backward(t, g, stats, ctx.contrast), None


def normalize(t, contrast=0.0):
    """Differentiable normalize_tensor on the device kernels (gradient to ``t``)."""
    return _Normalize.apply(t.contiguous(), float(contrast))


def adam_step(param, grad, exp_avg, exp_avg_sq, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    lib = N.lib()
    N.check(lib.dm_adam_step(N.ptr(param), N.ptr(grad), N.ptr(exp_avg), N.ptr(exp_avg_sq),
                             param.numel(), float(lr), float(beta1), float(beta2), float(eps),
                             N.ptr(step), N.stream_ptr(param.device)), "dm_adam_step")


# ---------------------------------------------------------------------------
# occupancy and volumetric IoU (evaluation of fits)

def voxelize(verts, faces, grid: FreqGrid) -> torch.Tensor:
    """uint8 occupancy of the closed mesh at the image sample positions of ``grid``."""
    N.require_cuda(verts, "verts", torch.float32)
    N.require_cuda(faces, "faces", torch.int64)
    lib = N.lib()
    occ = torch.empty(grid.shape, dtype=torch.uint8, device=verts.device)
    st = torch.zeros(1, dtype=torch.int32, device=verts.device)
    N.check(lib.dm_voxelize(N.ptr(verts), verts.shape[0], N.ptr(faces), faces.shape[0],
                            ctypes.byref(grid.cbox), N.ptr(occ), N.ptr(st),
                            N.stream_ptr(verts.device)), "dm_voxelize")
    return occ


def iou(a: torch.Tensor, b: torch.Tensor) -> float:
    """Intersection over union of two occupancy grids."""
    a, b = a.bool(), b.bool()
    inter = torch.logical_and(a, b).sum()
    union = torch.logical_or(a, b).sum()
    return float(inter) / max(float(union), 1.0)
