"""Preconditioned fitting: the reference notebook's "large steps" gradient filter.

The reference fit loop (``Examples/Gradient_Descent.ipynb`` cell 2) builds
``M = I + lambda * L`` with largesteps' ``compute_matrix`` (L the uniform mesh
Laplacian: degree on the diagonal, -1 per edge) and replaces the vertex gradient
by ``(M @ M)^-1 g`` every step (``CholeskySolver(M@M).solve``); its optimiser is
``AdamUniform``, and deltaMic's own ``optimize.py`` ships the same filter as the
dense ``inv(M) @ inv(M)`` (``compute_precondition_matrix``, optimize.py:207-212)
and ``VectorAdam`` (optimize.py:215-258).

Two forms of the same operator:

* dense (default up to 16,384 vertices): ``P = (M @ M)^-1`` formed once per
  topology on the GPU in float64 (a Cholesky factorisation and inverse of the dense
  SPD matrix -- set-up work, as the reference's ``torch.inverse``), stored as a
  padded float32 matrix and applied every step by the HBM-bound product
  ``dm_precond_apply``: ``4 nv^2`` bytes (420 MB at 10,242 vertices);
* sparse (``method="chebyshev"``, the default above that size): two Chebyshev
  solves with the sparse ``M`` (``dm_precond_chebyshev``, one launch per
  iteration), for the eigenvalue interval ``[1, 1 + lambda max_(i,j) (d_i + d_j)]``
  of M (the Laplacian's spectrum lies in ``[0, max over edges of the sum of the two
  degrees]``, Anderson and Morley 1985) and an iteration count from the Chebyshev
  error bound ``2 q^k`` for relative error ``tol``; ``O(nv)`` memory.

The optimiser step is ``dm_vector_adam_step``.
"""
from __future__ import annotations

import math

import torch

from . import _native as N

__all__ = ["uniform_laplacian", "laplacian_csr", "chebyshev_plan", "LargeStepsPreconditioner",
           "vector_adam_step"]


def uniform_laplacian(faces, nv: int, dtype=torch.float64, device="cuda") -> torch.Tensor:
    """Dense uniform Laplacian L = D - A of the mesh edges (each undirected edge once)."""
    f = torch.as_tensor(faces, device=device).long()
    e = torch.cat([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], 0)
    e = torch.sort(e, dim=1).values
    e = torch.unique(e, dim=0)
    L = torch.zeros(nv, nv, dtype=dtype, device=device)
    one = torch.ones(e.shape[0], dtype=dtype, device=device)
    L.index_put_((e[:, 0], e[:, 1]), -one, accumulate=True)
    L.index_put_((e[:, 1], e[:, 0]), -one, accumulate=True)
    deg = torch.zeros(nv, dtype=dtype, device=device)
    deg.index_add_(0, e[:, 0], one)
    deg.index_add_(0, e[:, 1], one)
    L += torch.diag(deg)
    return L


def laplacian_csr(faces, nv: int, device="cuda"):
    """CSR neighbour lists of the mesh edges: (rowp[nv+1], col) int32, row i holding
    the vertices that share an edge with i in ascending order; and the degrees."""
    f = torch.as_tensor(faces, device=device).long()
    e = torch.cat([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], 0)
    e = torch.unique(torch.sort(e, dim=1).values, dim=0)
    both = torch.cat([e, e[:, [1, 0]]], 0)
    key = both[:, 0] * nv + both[:, 1]
    both = both[torch.argsort(key)]
    deg = torch.bincount(both[:, 0], minlength=nv)
    rowp = torch.zeros(nv + 1, dtype=torch.int64, device=device)
    rowp[1:] = torch.cumsum(deg, 0)
    return rowp.to(torch.int32), both[:, 1].to(torch.int32).contiguous(), deg, e


def chebyshev_plan(deg, edges, lambda_: float, tol: float = 1e-6):
    """(lo, hi, iterations) of the Chebyshev solves with M = I + lambda L."""
    bound = float((deg[edges[:, 0]] + deg[edges[:, 1]]).max()) if edges.numel() else 0.0
    lo, hi = 1.0, 1.0 + float(lambda_) * bound
    kappa = hi / lo
    if kappa <= 1.0 + 1e-12:
        return lo, hi, 1
    q = (math.sqrt(kappa) - 1.0) / (math.sqrt(kappa) + 1.0)
    return lo, hi, max(1, int(math.ceil(math.log(2.0 / tol) / math.log(1.0 / q))))


class LargeStepsPreconditioner:
    """``apply(g)`` returns ``(M @ M)^-1 g`` with ``M = I + lambda_ * L``.

    ``method``: "dense" (the formed operator, ``nv * ceil(nv/4)*4 * 4`` bytes of
    device memory -- 420 MB at 10,242 vertices), "chebyshev" (sparse, ``O(nv)``)
    or "auto" (dense up to 16,384 vertices)."""

    DENSE_MAX_VERTS = 16384

    def __init__(self, faces, nv: int, lambda_: float = 50.0, device="cuda", method="auto",
                 tol: float = 1e-6):
        self.nv = int(nv)
        self.lambda_ = float(lambda_)
        self.device = torch.device(device)
        if method not in ("auto", "dense", "chebyshev"):
            raise ValueError("method must be 'auto', 'dense' or 'chebyshev'")
        if method == "auto":
            method = "dense" if self.nv <= self.DENSE_MAX_VERTS else "chebyshev"
        self.method = method
        if method == "chebyshev":
            self.rowp, self.col, deg, edges = laplacian_csr(faces, self.nv, self.device)
            self.lo, self.hi, self.iters = chebyshev_plan(deg, edges, self.lambda_, tol)
            self.work = torch.empty(12 * max(self.nv, 1), dtype=torch.float32,
                                    device=self.device)
            self.P = None
            return
        L = uniform_laplacian(faces, self.nv, torch.float64, self.device)
        M = torch.eye(self.nv, dtype=torch.float64, device=self.device) + self.lambda_ * L
        del L
        # (M M)^-1 = (M^-1)^2 with M SPD: one Cholesky factorisation
        C = torch.linalg.cholesky(M)
        Minv = torch.cholesky_inverse(C)
        del C, M
        P64 = Minv @ Minv
        del Minv
        self.ldp = (self.nv + 3) // 4 * 4
        self.P = torch.zeros(self.nv, self.ldp, dtype=torch.float32, device=self.device)
        self.P[:, :self.nv] = P64.float()
        del P64

    def apply(self, grad: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        N.require_cuda(grad, "grad", torch.float32)
        if grad.shape != (self.nv, 3):
            raise ValueError(f"grad must have shape [{self.nv}, 3]")
        out = torch.empty_like(grad) if out is None else out
        if self.method == "chebyshev":
            N.check(N.lib().dm_precond_chebyshev(
                N.ptr(self.rowp), N.ptr(self.col), self.nv, self.lambda_, self.lo, self.hi,
                self.iters, N.ptr(grad.contiguous()), N.ptr(out), N.ptr(self.work),
                N.stream_ptr(grad.device)), "dm_precond_chebyshev")
            return out
        N.check(N.lib().dm_precond_apply(N.ptr(self.P), self.nv, self.ldp, N.ptr(grad),
                                         N.ptr(out), N.stream_ptr(grad.device)),
                "dm_precond_apply")
        return out


def vector_adam_step(param, grad, exp_avg, exp_avg_norm_sq, step, lr, beta1=0.9, beta2=0.999,
                     eps=1e-8):
    """VectorAdam (optimize.py:215-258) on [nv, 3] parameters; ``step`` a device int64."""
    N.check(N.lib().dm_vector_adam_step(N.ptr(param), N.ptr(grad), N.ptr(exp_avg),
                                        N.ptr(exp_avg_norm_sq), param.shape[0], float(lr),
                                        float(beta1), float(beta2), float(eps), N.ptr(step),
                                        N.stream_ptr(param.device)), "dm_vector_adam_step")
