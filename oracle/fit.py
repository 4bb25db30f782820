"""Oracle: the preconditioned fit step -- TEST INFRASTRUCTURE ONLY.

Restates in numpy float64
* largesteps' ``compute_matrix`` (an external dependency of the reference,
  ``largesteps>=0.2.1`` in requirements.txt, absent here): ``M = I + lambda L`` with
  L the uniform Laplacian of the mesh -- per undirected edge -1 off the diagonal,
  the vertex valence on it (Nicolet, Jacobson, Jakob 2021, "Large Steps in Inverse
  Rendering of Geometry");
* the dense preconditioner of ``compute_precondition_matrix``
  (``deltamic/optimize.py:207-212``): ``inv(M) @ inv(M)``, which is what the
  notebook's ``CholeskySolver(M@M).solve`` applies;
* ``VectorAdam.step`` (``deltamic/optimize.py:225-258``, axis -1).
"""
from __future__ import annotations

import numpy as np


def uniform_laplacian(faces, nv):
    f = np.asarray(faces, np.int64)
    e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
    e = np.unique(np.sort(e, axis=1), axis=0)
    L = np.zeros((nv, nv))
    L[e[:, 0], e[:, 1]] -= 1.0
    L[e[:, 1], e[:, 0]] -= 1.0
    np.add.at(L, (e[:, 0], e[:, 0]), 1.0)
    np.add.at(L, (e[:, 1], e[:, 1]), 1.0)
    return L


def precondition_matrix(faces, nv, lambda_):
    """inv(M) @ inv(M), M = I + lambda L (optimize.py:207-212 with p = 2)."""
    M = np.eye(nv) + lambda_ * uniform_laplacian(faces, nv)
    Minv = np.linalg.inv(M)
    return Minv @ Minv


def vector_adam_step(p, grad, g1, g2, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One VectorAdam step on [nv, 3] arrays; returns (p, g1, g2, step) updated.
    ``g2`` holds the per-vertex second moment repeated over the 3 components, as
    the reference stores it."""
    step = step + 1
    g1 = b1 * g1 + (1 - b1) * grad
    nrm = np.linalg.norm(grad, axis=-1, keepdims=True)
    g2 = b2 * g2 + (1 - b2) * np.repeat(nrm * nrm, grad.shape[-1], axis=-1)
    m1 = g1 / (1 - b1 ** step)
    m2 = g2 / (1 - b2 ** step)
    p = p - lr * (m1 / (eps + np.sqrt(m2)))
    return p, g1, g2, step
