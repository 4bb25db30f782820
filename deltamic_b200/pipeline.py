"""Fused render-and-loss path: meshFT -> ifftn of ft * OTF -> |.| / normalize_tensor
/ loss and dL/dz -> fftn of dL/dz on the band -> meshFT adjoint.

Two implementations of the middle part, both on the GPU: the band-box render
(``ops.render_loss_bandbox``: separable DFTs pruned to the band's bounding box,
fused with the image loss; the default wherever the library serves the box) and
the dense one (the OTF multiply in the meshFT epilogue, cuFFT on the whole grid,
the fused image-loss kernels, cuFFT again).

This is the chain ``normalize_tensor(render_image_from_ftmesh(meshFT(V,F,c), OTF))``
of the reference fitting loop (``Examples/Gradient_Descent.ipynb`` cell 2) with
the dense complex spectrum kept resident: only band voxels of the spectrum are
ever written, so it is zeroed once per narrow band, not per step.
"""
from __future__ import annotations

import torch

from . import ops

__all__ = ["MeshRenderer"]


class MeshRenderer:
    """Renderer for one box: holds the frequency grid, the OTF and its narrow band."""

    def __init__(self, box_size, box_shape, narrowband_thresh=1e-5, device="cuda",
                 autotune=True, render_path="auto"):
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("MeshRenderer runs on CUDA devices only")
        self.grid = ops.FreqGrid(box_size, box_shape)
        self.shape = self.grid.shape
        self.thresh = float(narrowband_thresh)
        self.xi = self.grid.axes(torch.float32, self.device)
        c64 = dict(dtype=torch.complex64, device=self.device)
        self.spec = torch.zeros(self.shape, **c64)     # ft * OTF on the band, 0 elsewhere
        self.z = torch.empty(self.shape, **c64)        # ifftn(spec)
        self.G = torch.empty(self.shape, **c64)        # fftn(dL/dz)
        self.otf = None
        self.band = None
        self._sigma_key = None
        self.autotune = autotune
        self.variants = None
        if render_path not in ("auto", "bandbox", "dense"):
            raise ValueError("render_path must be 'auto', 'bandbox' or 'dense'")
        self.render_path = render_path
        self.bbox = None

    @property
    def numel(self) -> int:
        return self.grid.numel

    # -- PSF / band -----------------------------------------------------------
    def set_otf(self, otf: torch.Tensor) -> None:
        """Use ``otf`` (float32, box_shape) and recompute the narrow band."""
        self.otf = otf.detach().float().contiguous()
        self.band = ops.narrowband(self.otf, self.thresh)
        self.spec.zero_()
        self._sigma_key = None
        self.variants = None
        self.bbox = ops.BandBox(self.grid, self.band)
        if self.render_path == "bandbox" and not self.bbox.supported:
            raise RuntimeError(f"band box extent {self.bbox.extent} is not served by the "
                               "band-box render (axis-2 extent above 32 or tiles too large)")

    def set_sigma(self, sigma: torch.Tensor) -> None:
        """Gaussian OTF of ``sigma`` (psf.py:15-20) and its narrow band."""
        s = sigma.detach().float().contiguous()
        key = (s.data_ptr(), s._version)
        if key == self._sigma_key and self.otf is not None:
            return
        with torch.no_grad():
            otf = ops.gaussian_otf(s, *self.xi)
        self.set_otf(otf)
        self._sigma_key = key

    @property
    def use_bandbox(self) -> bool:
        """True when the render + loss go through the band-box kernels."""
        return (self.render_path != "dense" and self.bbox is not None
                and self.bbox.supported)

    def render_loss(self, ft, kind, target, contrast):
        """(loss[1], G) from the band's meshFT ``ft``: the loss of the normalised render
        and G = fftn(dL/dz) on the band, the cotangent of meshft_backward_list
        (grad_list with otf and scale = 1/numel)."""
        loss, _, G = ops.render_loss_bandbox(ft, self.band, self.bbox, self.otf, kind, target,
                                             contrast, want_grad=True)
        return loss, G

    @property
    def n_band(self) -> int:
        return 0 if self.band is None else int(self.band.numel())

    @property
    def n_eval(self) -> int:
        """Band frequencies the meshFT kernels evaluate (half of a symmetric band)."""
        return 0 if self.band is None else ops.band_eval_count(self.band)

    # -- forward only ----------------------------------------------------------
    @torch.no_grad()
    def render(self, verts, faces, coeff) -> torch.Tensor:
        """|ifftn(meshFT * OTF)| as a new float32 tensor (no normalisation)."""
        self._require_band()
        self.tune(verts, faces, coeff)
        ops.meshft_list(verts, faces, coeff, self.grid, self.band, otf=self.otf,
                        spectrum=self.spec)
        torch.fft.ifftn(self.spec, out=self.z)
        return self.z.abs()

    def loss(self, verts, faces, coeff, kind="sum", target=None, contrast=0.0, sigma=None,
             otf=None):
        """Differentiable loss of the normalised render.

        Gradients flow to verts, coeff, and either ``sigma`` (the renderer's OTF is
        then the Gaussian OTF of sigma) or ``otf`` (any OTF tensor of box_shape,
        e.g. ``psf.otf_from_psf(Gaussian_psf(...)())`` as in the reference notebook;
        the narrow band follows it)."""
        if sigma is not None and otf is not None:
            raise ValueError("pass sigma or otf, not both")
        if sigma is not None:
            self.set_sigma(sigma)
        else:
            sigma = torch.zeros(0, device=self.device)
        if otf is not None:
            if tuple(otf.shape) != tuple(self.shape):
                raise ValueError("otf must have shape box_shape")
            key = (otf.data_ptr(), otf._version)
            if key != getattr(self, "_otf_key", None) or self.otf is None:
                self.set_otf(otf)
                self._otf_key = key
            otf_in = otf
        else:
            otf_in = torch.zeros(0, device=self.device)
        self._require_band()
        ops._check_mesh(verts, faces, coeff)
        self.tune(verts, faces, coeff)
        return _RenderLoss.apply(verts.contiguous(), coeff.contiguous(), sigma, otf_in, self,
                                 faces.contiguous(), kind, target, float(contrast))

    def _require_band(self):
        if self.band is None:
            raise RuntimeError("call set_otf() or set_sigma() first")

    def tune(self, verts, faces, coeff):
        """Choose (once per size class) and apply the kernels' tile-shape variants."""
        from . import autotune
        self._require_band()
        if self.variants is None:
            if self.autotune:
                self.variants = autotune.tune(verts.detach().contiguous(), faces.contiguous(),
                                              coeff.detach().contiguous(), self.grid, self.band)
            else:
                self.variants = autotune.current()[:2]
        autotune.apply(self.variants)


class _RenderLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, verts, coeff, sigma, otf_in, r: MeshRenderer, faces, kind, target,
                contrast):
        ctx.bandbox = r.use_bandbox
        if ctx.bandbox:
            ft = ops.meshft_list(verts, faces, coeff, r.grid, r.band)
            loss, g = r.render_loss(ft, kind, target, contrast)
        else:
            ft = ops.meshft_list(verts, faces, coeff, r.grid, r.band, otf=r.otf, spectrum=r.spec)
            torch.fft.ifftn(r.spec, out=r.z)
            loss, _, g = ops.image_loss(r.z, kind, target, contrast, want_grad=True)
        ctx.save_for_backward(verts, coeff, faces, ft, g)
        ctx.r = r
        ctx.sigma_grad = sigma.numel() == 9 and ctx.needs_input_grad[2]
        ctx.otf_grad = otf_in.numel() > 0 and ctx.needs_input_grad[3]
        return loss.view(())

    @staticmethod
    def backward(ctx, gl):
        verts, coeff, faces, ft, g = ctx.saved_tensors
        r = ctx.r
        if ctx.bandbox:
            cot = dict(grad_list=g)
        else:
            torch.fft.fftn(g, out=r.G)
            cot = dict(grad_grid=r.G)
        gv, gc, go = ops.meshft_backward_list(
            verts, faces, coeff, r.grid, r.band, ft, otf=r.otf, scale=1.0 / r.numel,
            want_coeff=ctx.needs_input_grad[1], want_otf=ctx.sigma_grad or ctx.otf_grad,
            **cot)
        gv = gv * gl
        if gc is not None:
            gc = gc * gl
        gs = go_dense = None
        if ctx.sigma_grad:
            gs = ops.sigma_grad_dense(go, r.otf, *r.xi, band=r.band) * gl
        if ctx.otf_grad:  # the OTF enters the render on the band only
            go_dense = torch.zeros(r.shape, dtype=torch.float32, device=go.device)
            go_dense.view(-1)[r.band.long()] = go * gl
        return gv, gc, gs, go_dense, None, None, None, None, None
