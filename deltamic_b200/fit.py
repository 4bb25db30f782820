"""Gradient-descent fitting of a mesh to a 3D image (the loop of the reference's
``Examples/Gradient_Descent.ipynb`` cell 2, with plain Adam on the vertices).

``FitStep`` runs one iteration -- fused render + loss (``MeshRenderer``), adjoint,
Adam -- entirely on the GPU and, by default, replays it as one captured CUDA graph.

Checkpoints: ``FitStep.state_dict()`` / ``load_state_dict()`` hold the fit state
(vertices, Adam moments, step count, learning rate and betas), and
``save_fit_state`` / ``load_fit_state`` write and read it with ``torch.save``
together with the Faces_coeff and PSF sigma of the run (the reference notebook
saves the mesh with ``np.savez`` every 100 iterations,
Examples/Gradient_Descent.ipynb cell 2).  Loading copies into the step's own
tensors, so a captured graph keeps working.
"""
from __future__ import annotations

import torch

from . import _native as N
from . import ops
from .pipeline import MeshRenderer

__all__ = ["FitStep", "fit_mesh", "run_fit", "mesh_iou", "fit_state_dict",
           "load_fit_state_dict", "save_fit_state", "load_fit_state"]

_STATE_TENSORS = (("verts", "V"), ("adam_m", "m"), ("adam_v", "v"), ("step", "t"))


def fit_state_dict(step) -> dict:
    """CPU copies of a fit step's state: ``verts``, ``adam_m``, ``adam_v`` (per
    vertex for VectorAdam), ``step`` and the optimiser settings."""
    out = {k: getattr(step, a).detach().cpu().clone() for k, a in _STATE_TENSORS}
    out.update(lr=float(step.lr), betas=tuple(float(b) for b in step.betas), eps=float(step.eps),
               optimizer=str(step.optimizer))
    return out


def load_fit_state_dict(step, state: dict) -> None:
    """Copy a state from :func:`fit_state_dict` into the step's tensors in place
    (shapes must match; a graph captured on those tensors replays the loaded
    state)."""
    if str(state.get("optimizer", step.optimizer)) != str(step.optimizer):
        raise ValueError(f"state is for optimizer {state['optimizer']!r}, step uses "
                         f"{step.optimizer!r}")
    for k, a in _STATE_TENSORS:
        dst, src = getattr(step, a), state[k]
        if tuple(src.shape) != tuple(dst.shape):
            raise ValueError(f"{k}: state has shape {tuple(src.shape)}, step {tuple(dst.shape)}")
    settings = (float(state.get("lr", step.lr)), tuple(float(b) for b in
                state.get("betas", step.betas)), float(state.get("eps", step.eps)))
    if getattr(step, "graph", None) is not None and settings != (
            float(step.lr), tuple(float(b) for b in step.betas), float(step.eps)):
        # the captured graph holds the optimiser settings as launch arguments
        raise ValueError("the state's lr/betas/eps differ from this captured step's; "
                         "build the FitStep with the saved settings, then load")
    for k, a in _STATE_TENSORS:
        dst = getattr(step, a)
        dst.copy_(state[k].to(device=dst.device, dtype=dst.dtype))
    step.lr, step.betas, step.eps = settings


def save_fit_state(path, step, faces_coeff=None, sigma=None, **extra) -> None:
    """torch.save of the fit state, the run's Faces_coeff and sigma, and ``extra``."""
    state = fit_state_dict(step)
    if faces_coeff is not None:
        state["faces_coeff"] = faces_coeff.detach().cpu().clone()
    if sigma is not None:
        state["sigma"] = torch.as_tensor(sigma).detach().cpu().clone()
    state["extra"] = dict(extra)
    torch.save(state, path)


def load_fit_state(path, step=None) -> dict:
    """Read a file of :func:`save_fit_state`; with ``step``, load it into the step.
    Returns the saved dict (faces_coeff, sigma and extra included)."""
    state = torch.load(path, map_location="cpu", weights_only=False)
    if step is not None:
        load_fit_state_dict(step, state)
    return state


class FitStep:
    """One Adam step on ``verts`` minimising the loss of the normalised render.

    ``verts`` is updated in place (it is the optimised parameter).  The loss of the
    step (evaluated before the update, like ``loss.backward(); opt.step()``) is
    left in ``self.loss`` on the device.

    ``restore`` (optional, [nv, 3] float32 on the device): copied into ``verts`` at
    the start of every step, so every step renders the same mesh and does the same
    work (a step timed at one mesh state; the update is still computed and applied).
    """

    def __init__(self, renderer: MeshRenderer, verts, faces, coeff, target=None, kind="mse",
                 contrast=0.0, lr=1e-3, betas=(0.9, 0.999), eps=1e-8, graph=True,
                 precond=None, optimizer="adam", restore=None):
        ops._check_mesh(verts, faces, coeff)
        if restore is not None and (restore.shape != verts.shape or restore.dtype != verts.dtype
                                    or restore.device != verts.device):
            raise ValueError("restore must match verts in shape, dtype and device")
        self.restore = restore
        if renderer.band is None:
            raise RuntimeError("set the renderer's OTF first")
        self.r = renderer
        self.V = verts
        self.F = faces.contiguous()
        self.C = coeff.contiguous()
        self.target = target
        self.kind = kind
        self.contrast = float(contrast)
        self.lr, self.betas, self.eps = float(lr), betas, float(eps)
        if optimizer not in ("adam", "vector_adam"):
            raise ValueError("optimizer must be 'adam' or 'vector_adam'")
        self.optimizer = optimizer
        self.precond = precond  # e.g. precond.LargeStepsPreconditioner: g <- (M M)^-1 g
        self.m = torch.zeros_like(verts)
        self.v = (torch.zeros_like(verts) if optimizer == "adam"
                  else torch.zeros(verts.shape[0], dtype=verts.dtype, device=verts.device))
        self.gpre = torch.zeros_like(verts) if precond is not None else None
        self.t = torch.zeros(1, dtype=torch.int64, device=verts.device)
        self.loss = torch.zeros(1, dtype=torch.float32, device=verts.device)
        self.grad = torch.zeros_like(verts)
        renderer.tune(verts, self.F, self.C)
        self.graph = None
        self.launches_per_step = None
        if graph:
            self._capture()

    def _body(self):
        r = self.r
        if self.restore is not None:
            self.V.copy_(self.restore)
        if r.use_bandbox:
            ft = ops.meshft_list(self.V, self.F, self.C, r.grid, r.band)
            loss, G = r.render_loss(ft, self.kind, self.target, self.contrast)
            cot = dict(grad_list=G)
        else:
            ft = ops.meshft_list(self.V, self.F, self.C, r.grid, r.band, otf=r.otf,
                                 spectrum=r.spec)
            torch.fft.ifftn(r.spec, out=r.z)
            loss, _, gz = ops.image_loss(r.z, self.kind, self.target, self.contrast,
                                         want_grad=True)
            torch.fft.fftn(gz, out=r.G)
            cot = dict(grad_grid=r.G)
        self.loss.copy_(loss)
        gv, _, _ = ops.meshft_backward_list(self.V, self.F, self.C, r.grid, r.band, ft,
                                            otf=r.otf, scale=1.0 / r.numel, want_coeff=False,
                                            **cot)
        self.grad.copy_(gv)
        if self.precond is not None:
            gv = self.precond.apply(gv, out=self.gpre)
        if self.optimizer == "adam":
            ops.adam_step(self.V, gv, self.m, self.v, self.t, self.lr, self.betas[0],
                          self.betas[1], self.eps)
        else:
            from .precond import vector_adam_step
            vector_adam_step(self.V, gv, self.m, self.v, self.t, self.lr, self.betas[0],
                             self.betas[1], self.eps)

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

    def state_dict(self) -> dict:
        return fit_state_dict(self)

    def load_state_dict(self, state: dict) -> None:
        load_fit_state_dict(self, state)

    def __call__(self):
        if self.graph is not None:
            self.graph.replay()
        else:
            if self.launches_per_step is None:
                c0 = N.lib().dm_launch_count()
                self._body()
                self.launches_per_step = int(N.lib().dm_launch_count() - c0)
            else:
                self._body()
        return self.loss


def fit_mesh(renderer: MeshRenderer, verts0, faces, coeff, target, steps=300, lr=1e-3,
             kind="mse", contrast=0.0, graph=True, record_every=1):
    """Fit ``verts0`` to ``target`` (already normalised) with ``steps`` Adam steps.

    Returns ``(verts, losses)`` with the loss of every ``record_every``-th step."""
    V = verts0.detach().clone().contiguous()
    step = FitStep(renderer, V, faces, coeff, target, kind, contrast, lr, graph=graph)
    losses = torch.zeros(steps, device=V.device)
    for k in range(steps):
        step()
        losses[k] = step.loss[0]
    return V, losses[::record_every].cpu()


def run_fit(renderer: MeshRenderer, verts0, faces, coeff, target, steps=300, lr=1e-3,
            kind="mse", contrast=0.0, stop_at=None, graph=True, precond=None,
            optimizer="adam"):
    """Adam fit with per-step losses and device timing.

    Returns ``dict(verts, losses[steps_run], ms_total, steps_run, reached)``; with
    ``stop_at`` the fit stops at the first step whose loss is <= stop_at (checked
    on the host every step, so the timing includes one small read per step).
    """
    V = verts0.detach().clone().contiguous()
    step = FitStep(renderer, V, faces, coeff, target, kind, contrast, lr, graph=graph,
                   precond=precond, optimizer=optimizer)
    losses = torch.zeros(steps, device=V.device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    k, reached = 0, False
    for k in range(steps):
        step()
        losses[k] = step.loss[0]
        if stop_at is not None and float(step.loss[0]) <= stop_at:
            reached = True
            break
    e1.record()
    torch.cuda.synchronize()
    n = k + 1
    return dict(verts=V, losses=losses[:n].cpu(), ms_total=e0.elapsed_time(e1), steps_run=n,
                reached=reached)


def mesh_iou(verts_a, verts_b, faces, grid) -> float:
    """Volumetric IoU of two meshes with the same faces on ``grid``."""
    return ops.iou(ops.voxelize(verts_a.contiguous(), faces, grid),
                   ops.voxelize(verts_b.contiguous(), faces, grid))
