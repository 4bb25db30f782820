"""Batched render-and-fit: many cells (mesh, box, grid shape, PSF) per launch.

Each stage runs once for the whole batch: one meshFT forward launch over the
flattened (cell, frequency tile, face split) items, one adjoint launch over
(cell, face block, frequency chunk) items, and the render + normalise + loss
with its adjoint as the band-box DFTs of every cell, one launch per stage
(``dm_bandbox_batch_render_loss``).  ``render_path="dense"`` (or a cell whose
band box the line kernels do not serve, under ``"auto"``) renders with one
batched cuFFT per distinct grid shape and the batched image-loss kernels
instead.  Per-cell results are those of ``MeshRenderer`` on each cell alone.
"""
from __future__ import annotations

import ctypes
from collections import OrderedDict

import numpy as np
import torch

from . import _native as N
from . import ops

__all__ = ["BatchRenderer", "BatchFitStep"]


class BatchRenderer:
    """Cells ``i`` with ``boxes[i]`` ([3,2]) and ``shapes[i]`` (3 ints)."""

    def __init__(self, boxes, shapes, narrowband_thresh=1e-5, device="cuda",
                 render_path="auto", autotune=True):
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("BatchRenderer runs on CUDA devices only")
        if render_path not in ("auto", "bandbox", "dense"):
            raise ValueError("render_path must be 'auto', 'bandbox' or 'dense'")
        self.render_path = render_path
        self.autotune = autotune
        self.variants = None
        self.bb = None
        self.grids = [ops.FreqGrid(b, s) for b, s in zip(boxes, shapes)]
        self.ncells = len(self.grids)
        self.thresh = float(narrowband_thresh)
        # group cells by grid shape; each group is one contiguous [B, n0, n1, n2] block
        groups: "OrderedDict[tuple, list]" = OrderedDict()
        for i, g in enumerate(self.grids):
            groups.setdefault(g.shape, []).append(i)
        self.groups = []
        self.grid_offset = [0] * self.ncells
        off = 0
        for shape, ids in groups.items():
            n = int(np.prod(shape))
            for j, i in enumerate(ids):
                self.grid_offset[i] = off + j * n
            self.groups.append((shape, ids, off, len(ids)))
            off += n * len(ids)
        self.grid_elems = off
        c64 = dict(dtype=torch.complex64, device=self.device)
        self.spec = torch.zeros(off, **c64)
        self.z = torch.empty(off, **c64)
        self.G = torch.empty(off, **c64)
        self.otf = torch.empty(off, dtype=torch.float32, device=self.device)
        self.xi = [g.axes(torch.float32, self.device) for g in self.grids]
        self.band = None
        self.band_sizes = None
        self.batch = None
        self._desc = None
        self._topo = None
        self._mesh_key = None

    def cell_view(self, flat: torch.Tensor, i: int) -> torch.Tensor:
        """Cell ``i``'s grid inside a concatenated grid array, shaped ``shapes[i]``."""
        g = self.grids[i]
        o = self.grid_offset[i]
        return flat[o:o + g.numel].view(g.shape)

    def _group_view(self, flat, gi):
        shape, ids, off, count = self.groups[gi]
        return flat[off:off + count * int(np.prod(shape))].view(count, *shape)

    # -- PSFs and bands ---------------------------------------------------------
    def set_sigmas(self, sigmas) -> None:
        """Gaussian OTF per cell (psf.py:15-20) and the narrow bands."""
        bands = []
        with torch.no_grad():
            for i, s in enumerate(sigmas):
                s = torch.as_tensor(s, dtype=torch.float32, device=self.device).contiguous()
                o = ops.gaussian_otf(s, *self.xi[i])
                self.cell_view(self.otf, i).copy_(o)
                bands.append(ops.narrowband(o, self.thresh))
        self.band_sizes = [int(b.numel()) for b in bands]
        self.band_herm = [ops.band_is_hermitian(b) for b in bands]
        self.band = torch.cat(bands).contiguous()
        self.spec.zero_()
        self.batch = None
        self._plan_bandbox(bands)

    def _plan_bandbox(self, bands):
        """Band-box plan of every cell (one host sync per cell for its bounds)."""
        self.bb = None
        if self.render_path == "dense":
            return
        lib = N.lib()
        n = self.ncells
        cells = (N.DmCell * n)()
        flat = []
        ok = all(b.numel() > 0 for b in bands)
        for i, b in enumerate(bands):
            cells[i].n_band = self.band_sizes[i]
            cells[i].grid_offset = self.grid_offset[i]
            cells[i].box = ops.band_box(self.grids[i], self.band_herm[i])
            flat.extend(ops.band_bounds(b, self.grids[i]) if b.numel() else (0,) * 6)
        bounds = (ctypes.c_int32 * (6 * n))(*flat)
        size = ctypes.c_size_t(0)
        st = lib.dm_bandbox_batch_workspace_size(cells, bounds, n, ctypes.byref(size)) if ok \
            else N.DM_ERR_UNSUPPORTED
        if st != 0:
            if self.render_path == "bandbox":
                N.check(st, "dm_bandbox_batch_workspace_size")
            return
        self._bb_ws = torch.empty(max(int(size.value), 256), dtype=torch.uint8,
                                  device=self.device)
        self._bb_desc = torch.empty(lib.dm_bandbox_batch_desc_size(n), dtype=torch.uint8,
                                    device=self.device)
        plan = N.DmBandboxBatch()
        N.check(lib.dm_bandbox_batch_plan(cells, bounds, n, N.ptr(self._bb_desc),
                                          self._bb_desc.numel(), N.ptr(self._bb_ws),
                                          self._bb_ws.numel(), ctypes.byref(plan),
                                          N.stream_ptr(self.device)), "dm_bandbox_batch_plan")
        self.bb = plan

    @property
    def use_bandbox(self) -> bool:
        return self.bb is not None

    # -- meshes -----------------------------------------------------------------
    def set_meshes(self, verts_list, faces_list):
        """Concatenate the cells' meshes (faces keep cell-local indices) and plan."""
        if self.band is None:
            raise RuntimeError("call set_sigmas() first")
        nvs = [int(v.shape[0]) for v in verts_list]
        nts = [int(f.shape[0]) for f in faces_list]
        faces = torch.cat([torch.as_tensor(f, dtype=torch.int64, device=self.device)
                           for f in faces_list]).contiguous()
        for f, nv in zip(faces_list, nvs):
            ff = torch.as_tensor(f)
            if ff.numel() and (int(ff.min()) < 0 or int(ff.max()) >= nv):
                raise IndexError("face index out of range for its cell")
        cells = (N.DmCell * self.ncells)()
        for i in range(self.ncells):
            cells[i].nv, cells[i].nt, cells[i].n_band = nvs[i], nts[i], self.band_sizes[i]
            cells[i].grid_offset = self.grid_offset[i]
            cells[i].box = ops.band_box(self.grids[i], self.band_herm[i])
        self._cells = cells
        self.faces = faces
        self.nv, self.nt = nvs, nts
        self._plan()
        self.pairs = sum(nt * nb for nt, nb in zip(nts, self.band_sizes))
        # face*xi pairs the kernels evaluate (half of each mirror-symmetric band)
        self.eval_pairs = sum(nt * ((nb + 1) // 2 if h else nb)
                              for nt, nb, h in zip(nts, self.band_sizes, self.band_herm))
        return faces

    def _plan(self):
        """Plan the meshFT launches for the current tile variants (the launches use
        the variants the plan was made for), topology and workspaces."""
        lib = N.lib()
        self._desc = torch.empty(lib.dm_batch_desc_size(self.ncells), dtype=torch.uint8,
                                 device=self.device)
        self.batch = N.DmBatch()
        N.check(lib.dm_batch_plan(self._cells, self.ncells, N.ptr(self._desc),
                                  self._desc.numel(), ctypes.byref(self.batch),
                                  N.stream_ptr(self.device)), "dm_batch_plan")
        self._topo = torch.zeros(max(self.batch.topology_bytes, 256), dtype=torch.uint8,
                                 device=self.device)
        N.check(lib.dm_batched_topology_build(ctypes.byref(self.batch), N.ptr(self.faces),
                                              N.ptr(self._topo), self._topo.numel(),
                                              N.stream_ptr(self.device)),
                "dm_batched_topology_build")
        self._ws = {k: torch.zeros(max(int(getattr(self.batch, k)), 256), dtype=torch.uint8,
                                   device=self.device)
                    for k in ("fwd_workspace", "bwd_workspace", "image_workspace")}

    def tune(self, verts, coeff):
        """Time every forward and adjoint tile variant on this batch (a plan per
        variant) and keep the fastest; the batch is re-planned for them."""
        from . import autotune
        f0, b0, nf, nb = autotune.current()
        g = torch.ones(self.band.numel(), dtype=torch.complex64, device=self.device)

        def with_variant(v):
            autotune.apply(v)
            self._plan()

        def fwd():
            return self.forward_spectrum(verts, coeff, dense=False)

        ft = fwd()

        def bwd():
            return self.backward(verts, coeff, ft, want_coeff=False, grad_list=g)

        best_f = autotune._pick(nf, lambda v: with_variant((v, b0)), fwd, 2, trials=2)
        best_b = autotune._pick(nb, lambda v: with_variant((best_f, v)), bwd, 2, trials=2)
        self.variants = (best_f, best_b)
        with_variant(self.variants)
        autotune.apply((f0, b0))
        return self.variants

    # -- stages -----------------------------------------------------------------
    def forward_spectrum(self, verts, coeff, dense=True):
        """ft on the concatenated bands (complex64); with ``dense`` also ft * OTF
        scattered into the concatenated grids (the cuFFT path's input)."""
        lib = N.lib()
        ft = torch.empty(self.band.numel(), dtype=torch.complex64, device=self.device)
        w = self._ws["fwd_workspace"]
        N.check(lib.dm_batched_meshft_forward(
            ctypes.byref(self.batch), N.ptr(verts), N.ptr(self.faces), N.ptr(coeff),
            N.ptr(self.band), N.ptr(self.otf), N.ptr(ft), N.ptr(self.spec) if dense else None,
            N.ptr(w), w.numel(), N.stream_ptr(self.device)), "dm_batched_meshft_forward")
        return ft

    def render_loss_bandbox(self, ft, kind, target, contrast=0.0, want_grad=True,
                            want_image=False):
        """(losses[ncells], dL/dS on the concatenated bands | None, image | None) by
        the band-box DFTs of every cell."""
        lib = N.lib()
        losses = torch.empty(self.ncells, dtype=torch.float32, device=self.device)
        G = torch.empty_like(ft) if want_grad else None
        img = torch.empty(self.grid_elems, device=self.device) if want_image else None
        if kind == "mse":
            N.require_cuda(target, "target", torch.float32)
            if target.numel() != self.grid_elems:
                raise ValueError("target must hold every cell's grid")
        N.check(lib.dm_bandbox_batch_render_loss(
            ctypes.byref(self.bb), N.ptr(ft), N.ptr(self.band), N.ptr(self.otf),
            ops.LOSS_KINDS[kind], N.ptr(target) if kind == "mse" else None, float(contrast),
            N.ptr(losses), N.ptr(G), N.ptr(img), N.stream_ptr(self.device)),
            "dm_bandbox_batch_render_loss")
        return losses, G, img

    def device_error(self) -> int:
        """Status words of the band-box plan's cells (read and cleared; synchronous)."""
        flags = N._INT(0)
        if self.bb is not None:
            N.check(N.lib().dm_bandbox_batch_device_error(ctypes.byref(self.bb),
                                                          ctypes.byref(flags),
                                                          N.stream_ptr(self.device)),
                    "dm_bandbox_batch_device_error")
        return flags.value

    def inverse_fft(self):
        for gi in range(len(self.groups)):
            torch.fft.ifftn(self._group_view(self.spec, gi), dim=(-3, -2, -1),
                            out=self._group_view(self.z, gi))

    def adjoint_fft(self, gz):
        # norm="forward" divides by each cell's voxel count: the adjoint of ifftn
        for gi in range(len(self.groups)):
            torch.fft.fftn(self._group_view(gz, gi), dim=(-3, -2, -1), norm="forward",
                           out=self._group_view(self.G, gi))

    def image_loss(self, kind, target, contrast=0.0, want_grad=True, want_image=False):
        lib = N.lib()
        losses = torch.empty(self.ncells, dtype=torch.float32, device=self.device)
        gz = torch.empty_like(self.z) if want_grad else None
        img = torch.empty(self.grid_elems, device=self.device) if want_image else None
        w = self._ws["image_workspace"]
        N.check(lib.dm_batched_image_loss(
            ctypes.byref(self.batch), N.ptr(self.z), ops.LOSS_KINDS[kind], N.ptr(target),
            float(contrast), N.ptr(img), N.ptr(losses), N.ptr(gz), N.ptr(w), w.numel(),
            N.stream_ptr(self.device)), "dm_batched_image_loss")
        return losses, img, gz

    def backward(self, verts, coeff, ft, want_coeff=True, grad_list=None):
        """(grad_verts, grad_coeff | None) for the cotangent dL/dS: ``grad_list`` on
        the concatenated bands, or (default) the dense grids in ``self.G``."""
        lib = N.lib()
        gv = torch.empty_like(verts)
        gc = torch.empty_like(coeff) if want_coeff else None
        w = self._ws["bwd_workspace"]
        N.check(lib.dm_batched_meshft_backward(
            ctypes.byref(self.batch), N.ptr(verts), N.ptr(self.faces), N.ptr(coeff),
            N.ptr(self.band), N.ptr(grad_list), None if grad_list is not None else N.ptr(self.G),
            N.ptr(self.otf), 1.0, N.ptr(ft), N.ptr(self._topo), N.ptr(gv), N.ptr(gc), None,
            N.ptr(w), w.numel(), N.stream_ptr(self.device)), "dm_batched_meshft_backward")
        return gv, gc

    @torch.no_grad()
    def render(self, verts, coeff):
        """|ifftn(meshFT * OTF)| of every cell, concatenated (float32)."""
        if self.use_bandbox:
            ft = self.forward_spectrum(verts, coeff, dense=False)
            return self.render_loss_bandbox(ft, "sum", None, want_grad=False, want_image=True)[2]
        self.forward_spectrum(verts, coeff)
        self.inverse_fft()
        return self.z.abs()

    def loss(self, verts, coeff, kind="mse", target=None, contrast=0.0):
        """Sum over cells of each cell's normalised-image loss (differentiable)."""
        return _BatchLoss.apply(verts.contiguous(), coeff.contiguous(), self, kind, target,
                                float(contrast))


class _BatchLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, verts, coeff, r: BatchRenderer, kind, target, contrast):
        if r.use_bandbox:
            ft = r.forward_spectrum(verts, coeff, dense=False)
            losses, G, _ = r.render_loss_bandbox(ft, kind, target, contrast)
            ctx.save_for_backward(verts, coeff, ft, G)
        else:
            ft = r.forward_spectrum(verts, coeff)
            r.inverse_fft()
            losses, _, gz = r.image_loss(kind, target, contrast)
            ctx.save_for_backward(verts, coeff, ft, gz)
        ctx.bandbox = r.use_bandbox
        ctx.r = r
        return losses.sum()

    @staticmethod
    def backward(ctx, gl):
        verts, coeff, ft, g = ctx.saved_tensors
        r = ctx.r
        if ctx.bandbox:
            gv, gc = r.backward(verts, coeff, ft, want_coeff=ctx.needs_input_grad[1],
                                grad_list=g)
        else:
            r.adjoint_fft(g)
            gv, gc = r.backward(verts, coeff, ft, want_coeff=ctx.needs_input_grad[1])
        gv = gv * gl
        if gc is not None:
            gc = gc * gl
        return gv, gc, None, None, None, None


class BatchFitStep:
    """One Adam step on all cells' vertices (concatenated), replayed as a CUDA graph.

    ``restore`` (optional, like ``fit.FitStep``'s): copied into the vertices at the
    start of every step, so every step works on the same mesh state."""

    def __init__(self, r: BatchRenderer, verts, coeff, target, kind="mse", contrast=0.0,
                 lr=1e-3, betas=(0.9, 0.999), eps=1e-8, graph=True, restore=None):
        if restore is not None and (restore.shape != verts.shape or restore.dtype != verts.dtype
                                    or restore.device != verts.device):
            raise ValueError("restore must match verts in shape, dtype and device")
        self.restore = restore
        self.r, self.V, self.C, self.target = r, verts, coeff.contiguous(), target
        self.kind, self.contrast = kind, float(contrast)
        self.lr, self.betas, self.eps = float(lr), betas, float(eps)
        self.m = torch.zeros_like(verts)
        self.v = torch.zeros_like(verts)
        self.t = torch.zeros(1, dtype=torch.int64, device=verts.device)
        self.loss = torch.zeros(1, dtype=torch.float32, device=verts.device)
        self.cell_losses = torch.zeros(r.ncells, dtype=torch.float32, device=verts.device)
        self.graph = None
        self.launches_per_step = None
        if r.autotune and r.variants is None:
            r.tune(verts.detach().contiguous(), self.C)  # before any capture: it re-plans
        if graph:
            self._capture()

    def _body(self):
        r = self.r
        if self.restore is not None:
            self.V.copy_(self.restore)
        if r.use_bandbox:
            ft = r.forward_spectrum(self.V, self.C, dense=False)
            losses, G, _ = r.render_loss_bandbox(ft, self.kind, self.target, self.contrast)
            self.cell_losses.copy_(losses)
            torch.sum(losses, dim=0, keepdim=True, out=self.loss)
            gv, _ = r.backward(self.V, self.C, ft, want_coeff=False, grad_list=G)
        else:
            ft = r.forward_spectrum(self.V, self.C)
            r.inverse_fft()
            losses, _, gz = r.image_loss(self.kind, self.target, self.contrast)
            self.cell_losses.copy_(losses)
            torch.sum(losses, dim=0, keepdim=True, out=self.loss)
            r.adjoint_fft(gz)
            gv, _ = r.backward(self.V, self.C, ft, want_coeff=False)
        ops.adam_step(self.V, gv, self.m, self.v, self.t, self.lr, self.betas[0], self.betas[1],
                      self.eps)

    def _capture(self):
        state = [x.clone() for x in (self.V, self.m, self.v, self.t)]
        side = torch.cuda.Stream(device=self.V.device)
        side.wait_stream(torch.cuda.current_stream(self.V.device))
        with torch.cuda.stream(side):
            c0 = N.lib().dm_launch_count()
            self._body()
            self.launches_per_step = int(N.lib().dm_launch_count() - c0)
            self._body()
        torch.cuda.current_stream(self.V.device).wait_stream(side)
        for dst, src in zip((self.V, self.m, self.v, self.t), state):
            dst.copy_(src)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._body()

    def __call__(self):
        if self.graph is not None:
            self.graph.replay()
        else:
            self._body()
        return self.loss
