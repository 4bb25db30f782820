"""Oracle: surface + enclosed-volume ("autofluorescence") transform and its adjoint.

TEST INFRASTRUCTURE ONLY -- the checker for the CUDA path, never the product.

Restates ``fourier_from_mesh_narrowband_autofluorescence``
(``deltamic/render.py:228-318``) in numpy float64:

* ``trisar_k = 2 A_k / sum A`` with Heron areas (``render.py:202-218``, no
  Faces_coeff), ``nor_k = p0 x p1 + p1 x p2 + p2 x p0`` (``:217``),
  ``regvol = -sum_k p0 . (p1 x p2) / 6`` (``render.py:221-226``) and
  ``nor2 = nor regint / regvol`` (``:232``);
* per pair the divided-difference term ``F`` with the R1..R5 branches of
  ``:266-305`` (R1 strict ``<``, R2..R4 ``<=``, ``Seps = sqrt(1.19209e-7)``);
* ``ft(xi) = sum_k F_k (trisar_k + i xi.nor2_k / |xi|^2)`` (``:297-316``).

At xi = 0 (only on grids with every axis odd) the reference evaluates 0/0 and
returns NaN; here the volume term there is its limit, ``-regint`` (with
``F_k -> e^{-i xi.c_k}/2``, ``sum_k c_k . nor_k = sum_k p0.(p1 x p2) = -6 regvol``),
so ``ft(0) = 1 - regint``.

The adjoint is the chain rule of the same expression: the vertex phases through
``F`` with the complex weight, the Heron areas and ``sum A``, the normals, and
``regvol``; plus ``dL/dregint``.  ``g`` is the cotangent in PyTorch's convention
(``dL/dRe + i dL/dIm``).  Golden vectors made by the reference function itself
(``tests/golden/make_golden_volume.py``) pin this module.
"""
from __future__ import annotations

import numpy as np

from .meshft import SEPS_F32, _chunks, _default_threads, _pair, _pool_map


def _geometry(verts, faces):
    p = verts[faces]                                         # [nt, 3, 3]
    sides = p - p[:, [2, 0, 1]]
    ls = np.linalg.norm(sides, axis=2)
    hp = ls.sum(axis=1) / 2
    area = np.sqrt(hp * (hp - ls[:, 0]) * (hp - ls[:, 1]) * (hp - ls[:, 2]))
    nor = (np.cross(p[:, 0], p[:, 1]) + np.cross(p[:, 1], p[:, 2])
           + np.cross(p[:, 2], p[:, 0]))
    det = np.einsum("ij,ij->i", p[:, 0], np.cross(p[:, 1], p[:, 2]))
    regvol = -det.sum() / 6.0
    return p, area, nor, regvol


def _inv_norm2(xi):
    q = np.einsum("ij,ij->i", xi, xi)
    zero = q == 0.0
    inv = np.where(zero, 0.0, 1.0 / np.where(zero, 1.0, q))
    return inv, zero


def volume_forward(verts, faces, regint, xi_list, seps=SEPS_F32, chunk_pairs=2_000_000,
                   threads=None):
    """Return ``(ft[N], vol[N])``: the transform and its volume part per unit
    ``beta = regint / regvol`` (``ft = ft_surface + beta vol``)."""
    threads = _default_threads() if threads is None else threads
    verts = np.asarray(verts, np.float64)
    faces = np.asarray(faces, np.int64)
    xi = np.asarray(xi_list, np.float64)
    p, area, nor, regvol = _geometry(verts, faces)
    trisar = 2.0 * area / area.sum()
    beta = regint / regvol
    rows = max(1, chunk_pairs // max(1, len(faces)))

    def work(rng):
        s, e = rng
        x = xi[s:e]
        xiv = x @ verts.T
        F, _ = _pair(xiv[:, faces[:, 0]], xiv[:, faces[:, 1]], xiv[:, faces[:, 2]], seps, True,
                     grads=False)
        inv, zero = _inv_norm2(x)
        vol = 1j * (F * (x @ nor.T)).sum(axis=1) * inv
        vol[zero] = -regvol
        return F @ trisar + beta * vol, vol

    parts = _pool_map(work, _chunks(len(xi), rows), threads)
    if not parts:
        return np.zeros(0, np.complex128), np.zeros(0, np.complex128)
    return np.concatenate([a for a, _ in parts]), np.concatenate([b for _, b in parts])


def volume_backward(verts, faces, regint, xi_list, grad_list, seps=SEPS_F32,
                    chunk_pairs=1_000_000, threads=None):
    """Return ``(grad_verts[nv,3], grad_regint)`` for cotangent ``grad_list``."""
    threads = _default_threads() if threads is None else threads
    verts = np.asarray(verts, np.float64)
    faces = np.asarray(faces, np.int64)
    xi_all = np.asarray(xi_list, np.float64)
    g_all = np.asarray(grad_list, np.complex128)
    p, area, nor, regvol = _geometry(verts, faces)
    m = area.sum()
    trisar = 2.0 * area / m
    beta = regint / regvol
    rows = max(1, chunk_pairs // max(1, len(faces)))

    def work(rng):
        s, e = rng
        xi, g = xi_all[s:e], g_all[s:e]
        xiv = xi @ verts.T
        F, dF = _pair(xiv[:, faces[:, 0]], xiv[:, faces[:, 1]], xiv[:, faces[:, 2]], seps, True,
                      grads=True)
        inv, zero = _inv_norm2(xi)
        t = xi @ nor.T
        W = trisar[None, :] + 1j * beta * t * inv[:, None]
        cg = np.conj(g)[:, None]
        vol = 1j * (F * t).sum(axis=1) * inv
        g_beta = float(np.real(np.conj(g[~zero]) * vol[~zero]).sum())
        g0 = float(np.real(g[zero]).sum())
        r = np.real(cg * F).sum(axis=0)                              # dL/dtrisar_k
        nsum = (np.real(1j * cg * F) * inv[:, None]).T @ xi          # dL/dnor2_k [nt, 3]
        q = [np.real(cg * W * dF[c]).T @ xi for c in range(3)]       # phase terms [nt, 3]
        return g_beta, g0, r, nsum, q

    parts = _pool_map(work, _chunks(len(xi_all), rows), threads)
    g_beta = sum(x[0] for x in parts)
    g0 = sum(x[1] for x in parts)
    r = sum(x[2] for x in parts) if parts else np.zeros(len(faces))
    nsum = sum(x[3] for x in parts) if parts else np.zeros((len(faces), 3))
    s_a = float((trisar * r).sum())
    dlda = (2.0 * r - s_a) / m
    n = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    nhat = n / np.linalg.norm(n, axis=1, keepdims=True)
    dl_dregvol = -g_beta * beta / regvol
    gv = np.zeros_like(verts)
    for c in range(3):
        nx, pv = (c + 1) % 3, (c + 2) % 3
        q = sum(x[4][c] for x in parts) if parts else np.zeros((len(faces), 3))
        da = 0.5 * np.cross(nhat, p[:, pv] - p[:, nx])
        dn = beta * np.cross(p[:, nx] - p[:, pv], nsum)
        dv = dl_dregvol * (-np.cross(p[:, nx], p[:, pv]) / 6.0)
        np.add.at(gv, faces[:, c], q + dlda[:, None] * da + dn + dv)
    return gv, g_beta / regvol - g0
