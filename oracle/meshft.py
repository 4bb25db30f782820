"""Oracle: analytic triangle-mesh Fourier transform and its adjoint (numpy).

TEST INFRASTRUCTURE ONLY -- the checker for the CUDA path, never the product.

Restates, vectorised over (frequency x face) blocks:

* per-face areas: cross-product form ``|(b-a)x(c-a)|/2`` as in the reference CUDA
  host code (``deltamic/cpp/fourier3d_cuda_kernel.cu:38-51``) or Heron's formula as
  in the CPU path (``deltamic/render.py:21-33``); ``trisar = 2 A c / sum(A c)``
  (``render.py:38-41``, ``.cu:438-439``);
* the per-(face, xi) divided-difference term ``F`` with the branch structure
  R1..R5 of ``render.py:77-103`` / ``.cu:238-278`` (R1 = at least two phase
  differences within ``Seps``, then R2 |ab|, R3 |bc|, R4 |ca|, else R5);
* the partial derivatives dF/dx_a, dF/dx_b, dF/dx_c of ``.cu:73-233``;
* the vertex adjoint of ``Grad_Mesh_NUFT_kernel`` (``.cu:314-397``), i.e.
  ``dL/dv = sum_xi Re(conj(g) [sum_{k in v} (trisar_k dF_k/dx_v xi - F_k w_k)
  - ft gradmeshar_v])`` with ``w_k`` and ``gradmeshar`` from ``.cu:16-36`` and
  ``.cu:481-485``;
* the Faces_coeff gradient ``dL/dc_k = (A_k/M)(2 r_k - s)`` with
  ``r_k = sum_xi Re(conj(g) F_k)`` and ``s = sum_xi Re(conj(g) ft)``, which the
  reference obtains only through CPU autograd of ``render.py:21-41`` (derived from
  ``trisar_k = 2 A_k c_k / sum_j A_j c_j``).

``g`` is the cotangent in PyTorch's convention for complex outputs
(``dL/dRe + i dL/dIm``), so real-parameter gradients are ``Re(conj(g) dft)``.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

# render.py:64-65 uses sqrt(1.19209e-07) for both dtypes; the CUDA path uses
# sqrt(numeric_limits<scalar_t>::epsilon()) (.cu:454, :522).
SEPS_F32 = float(np.sqrt(np.float64(np.finfo(np.float32).eps)))
SEPS_F64 = float(np.sqrt(np.finfo(np.float64).eps))


def face_areas(verts, faces, coeff, method: str = "cross"):
    """Return ``(A[nt], M)``: per-face area times coefficient and their sum."""
    p = verts[faces]                       # [nt, 3, 3]
    if method == "cross":                  # .cu:38-40
        n = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
        a = 0.5 * np.linalg.norm(n, axis=1)
    elif method == "heron":                # render.py:21-33
        sides = p - p[:, [2, 0, 1]]
        ls = np.linalg.norm(sides, axis=2)
        hp = ls.sum(axis=1) / 2
        a = np.sqrt(hp * (hp - ls[:, 0]) * (hp - ls[:, 1]) * (hp - ls[:, 2]))
    else:
        raise ValueError(method)
    ac = coeff * a
    return ac, ac.sum()


def _masks(ab, bc, ca, seps, r1_strict):
    """Branch masks R1..R5 (render.py:77-95; .cu:250-272)."""
    lt = (lambda x: np.abs(x) < seps) if r1_strict else (lambda x: np.abs(x) <= seps)
    le = lambda x: np.abs(x) <= seps
    c1 = (lt(ab) & lt(bc)) | (lt(bc) & lt(ca)) | (lt(ca) & lt(ab))
    r1 = c1
    r2 = le(ab) & ~r1
    r3 = le(bc) & ~r1 & ~r2
    r4 = le(ca) & ~r1 & ~r2 & ~r3
    r5 = ~(r1 | r2 | r3 | r4)
    return r1, r2, r3, r4, r5


def _emi(x):
    return np.exp(-1j * x)


def pair_F(xa, xb, xc, seps=SEPS_F32, r1_strict=False):
    """F(x_a, x_b, x_c) for arrays of phases (render.py:97-103, .cu:238-278)."""
    F, _ = _pair(xa, xb, xc, seps, r1_strict, grads=False)
    return F


def pair_F_and_grads(xa, xb, xc, seps=SEPS_F32, r1_strict=False):
    """Return ``F, (dF/dxa, dF/dxb, dF/dxc)`` (.cu:73-233)."""
    return _pair(xa, xb, xc, seps, r1_strict, grads=True)


def _pair(xa, xb, xc, seps, r1_strict, grads):
    xa, xb, xc = np.broadcast_arrays(np.asarray(xa, np.float64),
                                     np.asarray(xb, np.float64),
                                     np.asarray(xc, np.float64))
    ab, bc, ca = xb - xa, xc - xb, xa - xc
    r1, r2, r3, r4, r5 = _masks(ab, bc, ca, seps, r1_strict)
    F = np.zeros(xa.shape, np.complex128)
    ga = np.zeros(xa.shape, np.complex128) if grads else None
    gb = np.zeros(xa.shape, np.complex128) if grads else None
    gc = np.zeros(xa.shape, np.complex128) if grads else None

    # R1: e^{-i mean}/2, every partial is -i F / 3
    if r1.any():
        xd = (xa[r1] + xb[r1] + xc[r1]) / 3.0
        f = _emi(xd) / 2.0
        F[r1] = f
        if grads:
            g = -1j * f / 3.0
            ga[r1] = g
            gb[r1] = g
            gc[r1] = g

    # R2..R4: two vertices merged at their midpoint d, third vertex o.
    # F = (i e_d + (e_d - e_o)/delta)/delta, delta = x_d - x_o;
    # each merged vertex gets gd = (e_d/2 - F)/delta, the other -iF - 2 gd.
    def merged(mask, xp, xq, xo, slot_o):
        if not mask.any():
            return
        xd = (xp[mask] + xq[mask]) / 2.0
        ed = _emi(xd)
        eo = _emi(xo[mask])
        delta = xd - xo[mask]
        f = (1j * ed + (ed - eo) / delta) / delta
        F[mask] = f
        if grads:
            gd = (ed / 2.0 - f) / delta
            go = -1j * f - 2.0 * gd
            outs = [ga, gb, gc]
            for s in range(3):
                outs[s][mask] = go if s == slot_o else gd

    merged(r2, xa, xb, xc, 2)
    merged(r3, xb, xc, xa, 0)
    merged(r4, xc, xa, xb, 1)

    # R5: generic divided difference (render.py:103) and its partials (.cu:122,176,230)
    if r5.any():
        a, b, c = xa[r5], xb[r5], xc[r5]
        ea, eb, ec = _emi(a), _emi(b), _emi(c)
        dab, dbc, dca = ab[r5], bc[r5], ca[r5]
        F[r5] = ea / (dab * dca) + eb / (dbc * dab) + ec / (dca * dbc)
        if grads:
            iab, ibc, ica = 1.0 / dab, 1.0 / dbc, 1.0 / dca
            ga[r5] = ((iab - ica - 1j) * ((ica * iab) * ea) + iab * ((iab * ibc) * eb)
                      - ica * ((ibc * ica) * ec))
            gb[r5] = ((ibc - iab - 1j) * ((iab * ibc) * eb) + ibc * ((ibc * ica) * ec)
                      - iab * ((ica * iab) * ea))
            gc[r5] = ((ica - ibc - 1j) * ((ibc * ica) * ec) + ica * ((ica * iab) * ea)
                      - ibc * ((iab * ibc) * eb))
    return F, ((ga, gb, gc) if grads else None)


def _chunks(n, size):
    return [(s, min(n, s + size)) for s in range(0, n, size)]


def _pool_map(fn, items, threads):
    if threads <= 1 or len(items) <= 1:
        return [fn(it) for it in items]
    with ThreadPoolExecutor(max_workers=threads) as ex:
        return list(ex.map(fn, items))


def _default_threads():
    return int(os.environ.get("DM_ORACLE_THREADS", "1"))


def meshft_forward(verts, faces, coeff, xi_list, seps=SEPS_F32, r1_strict=False,
                   area="cross", chunk_pairs=2_000_000, threads=None,
                   dtype=np.float64):
    """ft_list[m] = sum_k trisar_k F_k(xi_m)  (render.py:36-109, .cu:281-311).

    ``verts`` must already be shifted by ``box_size[:,0]`` (render.py:144,148).
    ``dtype=np.float32`` evaluates the phases and terms in single precision,
    mirroring the reference's float32 CPU path (used only as a timing baseline).
    """
    threads = _default_threads() if threads is None else threads
    verts = np.asarray(verts, dtype)
    coeff = np.asarray(coeff, dtype)
    xi_list = np.asarray(xi_list, dtype)
    faces = np.asarray(faces, np.int64)
    ac, m = face_areas(verts.astype(np.float64), faces, coeff.astype(np.float64), area)
    trisar = (2.0 * ac / m).astype(dtype)
    nt = len(faces)
    nxi = len(xi_list)
    if nt == 0 or nxi == 0:
        return np.zeros(nxi, np.complex128)
    rows = max(1, chunk_pairs // max(1, nt))
    cdt = np.complex64 if dtype == np.float32 else np.complex128

    def work(rng):
        s, e = rng
        xiv = xi_list[s:e] @ verts.T                       # [chunk, nv]
        xa, xb, xc = xiv[:, faces[:, 0]], xiv[:, faces[:, 1]], xiv[:, faces[:, 2]]
        if dtype == np.float32:
            F = _pair_f32(xa, xb, xc, np.float32(seps), r1_strict)
        else:
            F, _ = _pair(xa, xb, xc, seps, r1_strict, grads=False)
        return (F.astype(cdt) @ trisar.astype(cdt)).astype(np.complex128)

    parts = _pool_map(work, _chunks(nxi, rows), threads)
    return np.concatenate(parts)


def _pair_f32(xa, xb, xc, seps, r1_strict):
    """Single-precision evaluation of F with the reference's formulas (timing baseline)."""
    ab, bc, ca = xb - xa, xc - xb, xa - xc
    r1, r2, r3, r4, r5 = _masks(ab, bc, ca, seps, r1_strict)
    F = np.zeros(xa.shape, np.complex64)
    j = np.complex64(1j)
    if r1.any():
        F[r1] = np.exp(-j * ((xa[r1] + xb[r1] + xc[r1]) / np.float32(3))) / np.float32(2)
    for mask, xp, xq, xo in ((r2, xa, xb, xc), (r3, xb, xc, xa), (r4, xc, xa, xb)):
        if mask.any():
            xd = (xp[mask] + xq[mask]) / np.float32(2)
            ed = np.exp(-j * xd)
            delta = xd - xo[mask]
            F[mask] = (j * ed + (ed - np.exp(-j * xo[mask])) / delta) / delta
    a, b, c = xa[r5], xb[r5], xc[r5]
    F[r5] = (np.exp(-j * a) / (ab[r5] * ca[r5]) + np.exp(-j * b) / (bc[r5] * ab[r5])
             + np.exp(-j * c) / (ca[r5] * bc[r5]))
    return F


def _face_geometry(verts, faces, coeff):
    """trisar, w[nt,3,3] and gradmeshar[nv,3] (.cu:16-36, :481-485), float64."""
    p = verts[faces]
    n = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    nn = np.linalg.norm(n, axis=1)
    a = 0.5 * nn
    nhat = n / nn[:, None]
    ac = coeff * a
    m = ac.sum()
    w = np.empty((len(faces), 3, 3))
    w[:, 0] = np.cross(p[:, 2] - p[:, 1], nhat)
    w[:, 1] = np.cross(p[:, 0] - p[:, 2], nhat)
    w[:, 2] = np.cross(p[:, 1] - p[:, 0], nhat)
    w *= coeff[:, None, None] / m
    gradmeshar = np.zeros((len(verts), 3))
    for j in range(3):
        np.add.at(gradmeshar, faces[:, j], -w[:, j] / 2.0)
    trisar = 2.0 * ac / m
    return trisar, w, gradmeshar, a, m


def meshft_backward(verts, faces, coeff, xi_list, grad_list, ft_list,
                    seps=SEPS_F32, r1_strict=False, chunk_pairs=1_000_000,
                    threads=None):
    """Vertex and Faces_coeff gradients for cotangent ``grad_list`` on the band.

    Returns ``(grad_verts[nv,3], grad_coeff[nt])``.  ``verts`` shifted as in
    :func:`meshft_forward`.
    """
    threads = _default_threads() if threads is None else threads
    verts = np.asarray(verts, np.float64)
    coeff = np.asarray(coeff, np.float64)
    xi_list = np.asarray(xi_list, np.float64)
    faces = np.asarray(faces, np.int64)
    g = np.asarray(grad_list, np.complex128)
    ft = np.asarray(ft_list, np.complex128)
    nt, nv, nxi = len(faces), len(verts), len(xi_list)
    trisar, w, gradmeshar, a, m = _face_geometry(verts, faces, coeff)
    if nxi == 0:
        return np.zeros((nv, 3)), np.zeros(nt)
    rows = max(1, chunk_pairs // max(1, nt))

    def work(rng):
        s, e = rng
        xi = xi_list[s:e]
        xiv = xi @ verts.T
        xa, xb, xc = xiv[:, faces[:, 0]], xiv[:, faces[:, 1]], xiv[:, faces[:, 2]]
        F, (ga, gb, gc) = _pair(xa, xb, xc, seps, r1_strict, grads=True)
        cg = np.conj(g[s:e])[:, None]
        r = np.real(cg * F).sum(axis=0)                          # [nt]
        q = np.empty((nt, 3, 3))
        for corner, d in enumerate((ga, gb, gc)):
            z = np.real(cg * d)                                  # [chunk, nt]
            q[:, corner, :] = z.T @ xi                           # sum_xi z xi_j
        return r, q

    parts = _pool_map(work, _chunks(nxi, rows), threads)
    r = sum(p[0] for p in parts)
    q = sum(p[1] for p in parts)
    s = float(np.real(np.conj(g) * ft).sum())
    contrib = trisar[:, None, None] * q - r[:, None, None] * w   # [nt, 3(corner), 3]
    gv = -s * gradmeshar
    for corner in range(3):
        np.add.at(gv, faces[:, corner], contrib[:, corner])
    gcoef = (a / m) * (2.0 * r - s)
    return gv, gcoef
