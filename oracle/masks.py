"""Oracle: segmentation masks of ``deltamic/mask_creation.py`` (numpy + scipy).

TEST INFRASTRUCTURE ONLY -- the checker for the CUDA path, never the product.

The reference builds both masks on trimesh (``trimesh>=3.10.2``,
``requirements.txt``), which is absent here, so its mask functions cannot be run
and this restatement is parity-unpinned against the reference itself; its trimesh
parts restate trimesh's published algorithms:

* ``subdivide_to_size`` -- ``trimesh.remesh.subdivide_to_size``: every pass splits
  each face with an edge longer than ``max_edge`` into four at its edge midpoints
  (``(a + b) / 2``); faces whose edges all fit are final.  The vertices of the final
  faces are the point set the semantic mask samples (done per face here, which
  gives the same set as trimesh's batch passes);
* ``semantic_mask`` -- ``create_semantic_segmentation_mask`` (``mask_creation.py:
  208-222``): 1 at the grid point (``create_coords``, ``:195-205``) nearest to each
  such vertex (scipy ``KDTree``), returned flat as the reference does;
* ``instance_mask`` -- ``create_instance_segmentation_mask`` (``:225-266``): faces
  reordered so the larger label comes first (``reorder_faces``, ``:49-53``), every
  face split four-way ``k`` times (``subdivide_with_materials``, ``:60-176``, with
  ``k = min(max(ceil(log2(longest / dmax)) - 2, 0), 3)`` and ``longest`` the
  reference's ``compute_max_size_edges``, ``:22-30``), then for every grid point
  the nearest child centroid (KDTree) and the label on the side of its normal the
  point lies on, plus one.
"""
from __future__ import annotations

import numpy as np
from scipy.spatial import KDTree


def create_coords(box_shape, box_size):
    nx, ny, nz = (int(v) for v in box_shape)
    X = np.linspace(box_size[0, 0], box_size[0, 1], nx)
    Y = np.linspace(box_size[1, 0], box_size[1, 1], ny)
    Z = np.linspace(box_size[2, 0], box_size[2, 1], nz)
    gx, gy, gz = np.meshgrid(X, Y, Z, indexing="ij")
    return np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)


def _split(a, b, c):
    ab, bc, ca = (a + b) / 2, (b + c) / 2, (c + a) / 2
    return [(a, ab, ca), (ab, b, bc), (ca, bc, c), (ab, bc, ca)]


def subdivide_to_size(verts, faces, max_edge, max_iter):
    """Vertices of the final faces of trimesh's size-limited subdivision."""
    out = []
    for f in faces[:, :3]:
        stack = [(verts[f[0]], verts[f[1]], verts[f[2]], 0)]
        while stack:
            a, b, c, depth = stack.pop()
            e = [np.sqrt(((q - p) ** 2).sum()) for p, q in ((a, b), (b, c), (c, a))]
            if max(e) > max_edge:
                if depth >= max_iter:
                    raise ValueError("max_iter exceeded")
                stack.extend(t + (depth + 1,) for t in _split(a, b, c))
            else:
                out.extend([a, b, c])
    return np.array(out)


def semantic_mask(verts, faces, box_shape, box_size):
    box_shape = np.asarray(box_shape)
    dmax = np.amin((box_size[:, 1] - box_size[:, 0]) / box_shape)
    P = verts[faces[:, :3]]
    longest = np.linalg.norm(np.concatenate([P[:, 1] - P[:, 0], P[:, 2] - P[:, 1],
                                             P[:, 0] - P[:, 2]]), axis=1).max()
    max_iter = max(int(np.ceil(np.log2(longest / dmax))), 0) * 2 + 1
    pts = subdivide_to_size(verts, faces, dmax, max_iter)
    _, idx = KDTree(create_coords(box_shape, box_size)).query(pts)
    m = np.zeros(int(np.prod(box_shape)))
    m[idx] = 1
    return m


def instance_mask(verts, faces, box_shape, box_size):
    box_shape = np.asarray(box_shape)
    F = faces.copy()
    swap = F[:, 3] < F[:, 4]
    F[swap] = F[swap][:, [0, 2, 1, 4, 3]]
    dmax = np.amin((box_size[:, 1] - box_size[:, 0]) / box_shape)
    P = verts[F[:, :3]]
    e = np.hstack((P[:, 1] - P[:, 0], P[:, 2] - P[:, 1], P[:, 2] - P[:, 1]))
    longest = np.linalg.norm(e, axis=1).max()
    k = min(max(int(np.ceil(np.log2(longest / dmax))) - 2, 0), 3)
    tris = [(verts[f[0]], verts[f[1]], verts[f[2]], f[3], f[4]) for f in F]
    for _ in range(k):
        tris = [t + (l1, l2) for a, b, c, l1, l2 in tris for t in _split(a, b, c)]
    cen = np.array([(a + b + c) / 3 for a, b, c, _, _ in tris])
    nrm = np.array([np.cross(b - a, c - b) for a, b, c, _, _ in tris])
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    lab = np.array([(l1, l2) for *_, l1, l2 in tris], np.float64)
    pts = create_coords(box_shape, box_size)
    _, idx = KDTree(cen).query(pts)
    dot = ((cen[idx] - pts) * nrm[idx]).sum(axis=1)
    side = ((-np.sign(dot) + 1) / 2).astype(int)
    return lab[idx, side].reshape(*box_shape) + 1
