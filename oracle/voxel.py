"""Oracle: mesh occupancy on a grid -- TEST INFRASTRUCTURE ONLY.

``occupancy_parity`` restates the voxelizer's column ray-parity rule in numpy;
``occupancy_winding`` is an independent check by the generalised winding number
(sum of signed solid angles / 4 pi, Van Oosterom-Strackee), usable on small grids.
Sample positions are lo + (i, j, k) L / n, as the rendered image's.
"""
from __future__ import annotations

import numpy as np


def grid_points(box, shape):
    box = np.asarray(box, np.float64)
    axes = [box[d, 0] + np.arange(shape[d]) * (box[d, 1] - box[d, 0]) / shape[d]
            for d in range(3)]
    return axes


def occupancy_parity(verts, faces, box, shape):
    box = np.asarray(box, np.float64)
    ax = grid_points(box, shape)
    L0, L1 = box[0, 1] - box[0, 0], box[1, 1] - box[1, 0]
    px = box[0, 0] + (np.arange(shape[0]) + 0.3819660113e-6) * L0 / shape[0]
    py = box[1, 0] + (np.arange(shape[1]) + 0.6180339887e-6) * L1 / shape[1]
    P = np.asarray(verts, np.float64)[np.asarray(faces)]
    occ = np.zeros(shape, np.uint8)
    X, Y = np.meshgrid(px, py, indexing="ij")
    X, Y = X.ravel(), Y.ravel()
    crossings = [[] for _ in range(len(X))]
    for a, b, c in P:
        d = (b[0] - a[0]) * (c[1] - a[1]) - (c[0] - a[0]) * (b[1] - a[1])
        if d == 0:
            continue
        w1 = ((X - a[0]) * (c[1] - a[1]) - (c[0] - a[0]) * (Y - a[1])) / d
        w2 = ((b[0] - a[0]) * (Y - a[1]) - (X - a[0]) * (b[1] - a[1])) / d
        w0 = 1 - w1 - w2
        hit = np.flatnonzero((w0 >= 0) & (w1 >= 0) & (w2 >= 0))
        z = w0[hit] * a[2] + w1[hit] * b[2] + w2[hit] * c[2]
        for h, zz in zip(hit, z):
            crossings[h].append(zz)
    zs = ax[2]
    for col, cr in enumerate(crossings):
        if not cr:
            continue
        cr = np.sort(cr)
        below = np.searchsorted(cr, zs, side="left")
        occ.reshape(-1, shape[2])[col] = (below & 1).astype(np.uint8)
    return occ


def occupancy_winding(verts, faces, box, shape):
    ax = grid_points(box, shape)
    Q = np.stack(np.meshgrid(*ax, indexing="ij"), -1).reshape(-1, 3)
    P = np.asarray(verts, np.float64)[np.asarray(faces)]
    w = np.zeros(len(Q))
    for a, b, c in P:
        A, B, C = a - Q, b - Q, c - Q
        la, lb, lc = (np.linalg.norm(x, axis=1) for x in (A, B, C))
        num = np.einsum("ij,ij->i", A, np.cross(B, C))
        den = (la * lb * lc + np.einsum("ij,ij->i", A, B) * lc
               + np.einsum("ij,ij->i", B, C) * la + np.einsum("ij,ij->i", C, A) * lb)
        w += 2 * np.arctan2(num, den)
    return (np.abs(w / (4 * np.pi)) > 0.5).astype(np.uint8).reshape(shape)
