"""The fit loop's gradient filter and optimiser under the reference's names
(optimize.py:207-258), on this library's kernels.

* ``compute_precondition_matrix(Verts, Faces, lambda_)`` -- the dense
  ``inv(M) @ inv(M)`` with ``M = I + lambda_ * L`` (L the uniform Laplacian, as
  largesteps' ``compute_matrix`` builds it), formed in float64 by one Cholesky
  factorisation and returned in ``Verts``' dtype and device.
* ``VectorAdam(params, lr, betas, eps, axis)`` -- a ``torch.optim.Optimizer`` whose
  step runs ``dm_vector_adam_step`` (axis -1 on [nv, 3] float32 CUDA parameters:
  one second moment per vertex from the squared gradient norm) or ``dm_adam_step``
  (``axis=None``: elementwise Adam, float32 CUDA parameters).  The reference keeps
  the per-vertex second moment repeated over the three coordinates; here it is
  stored once per vertex (the update is the same).  A state in the reference's
  layout (``step`` a Python int, ``g2`` repeated per coordinate, e.g. from the
  reference optimiser's ``state_dict``) is converted on the next step; a state
  of any other shape raises ``ValueError``.

The reference module's Laplacian regularisers are not part of this library.
"""
from __future__ import annotations

import torch

from . import _native as N
from . import ops
from .precond import uniform_laplacian, vector_adam_step

__all__ = ["compute_precondition_matrix", "VectorAdam"]


def compute_precondition_matrix(Verts, Faces, lambda_):
    nv = int(Verts.shape[0])
    L = uniform_laplacian(Faces, nv, torch.float64, Verts.device)
    M = torch.eye(nv, dtype=torch.float64, device=Verts.device) + float(lambda_) * L
    Minv = torch.cholesky_inverse(torch.linalg.cholesky(M))
    return (Minv @ Minv).to(Verts.dtype)


def _adopt_state(state, p, vector):
    """Bring a loaded optimiser state into this module's layout in place: the
    reference keeps ``step`` as a Python int and, with an axis, ``g2`` as [nv, 3]
    (the per-vertex value repeated over the coordinates, optimize.py:236-251)."""
    if set(state) != {"step", "g1", "g2"}:
        raise ValueError(f"VectorAdam state has keys {sorted(state)}, expected step, g1, g2")
    step = state["step"]
    if not torch.is_tensor(step):
        step = torch.tensor([int(step)], dtype=torch.int64)
    state["step"] = step.reshape(1).to(device=p.device, dtype=torch.int64).contiguous()
    g1, g2 = state["g1"], state["g2"]
    if tuple(g1.shape) != tuple(p.shape):
        raise ValueError(f"VectorAdam g1 has shape {tuple(g1.shape)}, parameter {tuple(p.shape)}")
    state["g1"] = g1.to(device=p.device, dtype=p.dtype).contiguous()
    if vector and tuple(g2.shape) == tuple(p.shape):
        g2 = g2[:, 0]  # reference layout: the per-vertex moment repeated per coordinate
    want = (p.shape[0],) if vector else tuple(p.shape)
    if tuple(g2.shape) != want:
        raise ValueError(f"VectorAdam g2 has shape {tuple(g2.shape)}, expected {want}")
    state["g2"] = g2.to(device=p.device, dtype=p.dtype).contiguous()


class VectorAdam(torch.optim.Optimizer):
    def __init__(self, params, lr=0.1, betas=(0.9, 0.999), eps=1e-8, axis=-1):
        defaults = dict(lr=lr, betas=betas, eps=eps, axis=axis)
        super().__init__(params, defaults)

    @torch.no_grad()
    def step(self, closure=None):
        loss = None
        if closure is not None:
            with torch.enable_grad():
                loss = closure()
        for group in self.param_groups:
            b1, b2 = group["betas"]
            axis = group["axis"]
            for p in group["params"]:
                if p.grad is None:
                    continue
                N.require_cuda(p, "param", torch.float32)
                if not p.is_contiguous():
                    raise ValueError("VectorAdam needs contiguous parameters")
                grad = p.grad.contiguous()
                state = self.state[p]
                vector = axis is not None
                if vector and (p.dim() != 2 or p.shape[1] != 3 or axis not in (-1, 1)):
                    raise NotImplementedError(
                        "VectorAdam with an axis runs on [nv, 3] vertex arrays (axis -1)")
                if len(state) == 0:
                    state["step"] = torch.zeros(1, dtype=torch.int64, device=p.device)
                    state["g1"] = torch.zeros_like(p)
                    state["g2"] = (torch.zeros(p.shape[0], dtype=p.dtype, device=p.device)
                                   if vector else torch.zeros_like(p))
                else:
                    _adopt_state(state, p, vector)
                if vector:
                    vector_adam_step(p, grad, state["g1"], state["g2"], state["step"],
                                     group["lr"], b1, b2, group["eps"])
                else:
                    ops.adam_step(p, grad, state["g1"], state["g2"], state["step"],
                                  group["lr"], b1, b2, group["eps"])
        return loss
