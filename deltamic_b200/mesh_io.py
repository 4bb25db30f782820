"""Mesh files at the two ends of the fitting pipeline and the reference's mesh
assembly helpers.

* Wavefront ``.obj`` (the reference loads ``data/mesh/*.obj`` with
  ``trimesh.load``, ``Examples/Gradient_Descent.ipynb`` cell 1): ``read_obj``
  returns the file's ``v`` positions and the vertex indices of its ``f`` records
  (``i``, ``i/t``, ``i//n``, ``i/t/n`` forms; 1-based or negative indices; polygons
  split into fans from their first vertex).  With ``merge=True`` (trimesh's default
  processing) vertices whose coordinates agree to 8 decimals become one, the
  survivors kept in order of first appearance.
* Multitracker ``.rec`` (``data/mesh/*.rec``): a vertex count, one ``x y z`` line
  per vertex, a face count, then one ``a b c l1 l2`` line per face -- three 0-based
  vertex indices and the material labels on either side (the reference reads it
  with an external package's ``open_mesh_multitracker``,
  ``Examples/.ipynb_checkpoints/Example_multimaterial-checkpoint.ipynb``).
* ``create_initial_mesh_from_points_mm`` (``deltamic/mesh_utilities.py:28-48``): one
  subdivided sphere per point, merged with region labels.
* ``combine_all_verts_faces`` / ``combine_all_verts_faces_mm``
  (``deltamic/mesh_utilities.py:8-25``): concatenation of several meshes with the
  face indices offset.

Host-side file handling (text parsing and formatting with numpy); the meshes it
returns are numpy arrays ready for ``torch.tensor(..., device="cuda")``.
"""
from __future__ import annotations

import numpy as np

__all__ = ["read_obj", "write_obj", "read_rec", "write_rec", "combine_all_verts_faces",
           "combine_all_verts_faces_mm", "create_initial_mesh_from_points_mm"]


def _obj_index(tok: str, nv: int) -> int:
    i = int(tok.split("/")[0])
    if i == 0:
        raise ValueError("OBJ vertex indices start at 1")
    return i - 1 if i > 0 else nv + i


def read_obj(path, merge: bool = True):
    """``(verts[nv,3] float64, faces[nt,3] int64)`` of an OBJ file."""
    verts, faces = [], []
    with open(path) as fh:
        for line in fh:
            parts = line.split()
            if not parts:
                continue
            if parts[0] == "v":
                verts.append([float(parts[1]), float(parts[2]), float(parts[3])])
            elif parts[0] == "f":
                idx = [_obj_index(t, len(verts)) for t in parts[1:]]
                if len(idx) < 3:
                    raise ValueError(f"face with {len(idx)} vertices in {path}")
                for k in range(1, len(idx) - 1):
                    faces.append([idx[0], idx[k], idx[k + 1]])
    v = np.asarray(verts, np.float64).reshape(-1, 3)
    f = np.asarray(faces, np.int64).reshape(-1, 3)
    if len(f) and (f.min() < 0 or f.max() >= len(v)):
        raise ValueError(f"face index out of range in {path}")
    if merge and len(v):
        key = np.round(v, 8)
        _, first, inv = np.unique(key, axis=0, return_index=True, return_inverse=True)
        inv = inv.reshape(-1)
        order = np.argsort(first, kind="stable")       # survivors in order of appearance
        rank = np.empty_like(order)
        rank[order] = np.arange(len(order))
        v = v[first[order]]
        f = rank[inv][f]
    return v, f


def write_obj(path, verts, faces):
    """Write ``v`` and 1-based ``f`` records."""
    v = np.asarray(verts, np.float64)
    f = np.asarray(faces, np.int64)[:, :3] + 1
    with open(path, "w") as fh:
        fh.write("".join(f"v {a!r} {b!r} {c!r}\n" for a, b, c in v.tolist()))
        fh.write("".join(f"f {a} {b} {c}\n" for a, b, c in f.tolist()))


def read_rec(path):
    """``(verts[nv,3] float64, faces[nt,5] int64)`` of a multitracker file: columns
    0-2 vertex indices, 3-4 the material labels on either side of the face."""
    with open(path) as fh:
        tok = fh.read().split()
    nv = int(tok[0])
    v = np.asarray(tok[1:1 + 3 * nv], np.float64).reshape(nv, 3)
    p = 1 + 3 * nv
    nt = int(tok[p])
    f = np.asarray(tok[p + 1:p + 1 + 5 * nt], np.int64).reshape(nt, 5)
    if len(tok) != p + 1 + 5 * nt:
        raise ValueError(f"{path}: {len(tok) - (p + 1)} face fields for {nt} faces of 5")
    if nt and (f[:, :3].min() < 0 or f[:, :3].max() >= nv):
        raise ValueError(f"face index out of range in {path}")
    return v, f


def write_rec(path, verts, faces):
    """Write a multitracker file (``faces`` [nt,5]: indices and two labels)."""
    v = np.asarray(verts, np.float64)
    f = np.asarray(faces, np.int64)
    if f.ndim != 2 or f.shape[1] != 5:
        raise ValueError("faces must have shape [nt, 5]")
    with open(path, "w") as fh:
        fh.write(f"{len(v)}\n")
        fh.write("".join(f"{a!r} {b!r} {c!r}\n" for a, b, c in v.tolist()))
        fh.write(f"{len(f)}\n")
        fh.write("".join(" ".join(str(x) for x in row) + "\n" for row in f.tolist()))


def combine_all_verts_faces(All_verts, All_faces):
    """Stack meshes, offsetting each mesh's face indices by the vertices before it
    (mesh_utilities.py:18-25; like the reference, the face arrays are offset in
    place)."""
    total = 0
    for i in range(1, len(All_faces)):
        total += len(All_verts[i - 1])
        All_faces[i] += total
    return np.vstack(All_verts), np.vstack(All_faces)


def combine_all_verts_faces_mm(All_verts, All_faces):
    """The same for faces carrying material labels: only columns 0-2 are offset, and
    the faces come back as int32 (mesh_utilities.py:8-15)."""
    total = 0
    for i in range(1, len(All_faces)):
        total += len(All_verts[i - 1])
        All_faces[i][:, :3] += total
    return np.vstack(All_verts), np.vstack(All_faces).astype(np.int32)


def create_initial_mesh_from_points_mm(points, n_subdivisions=3, threshold_dist=0.9):
    """One sphere per point, merged into a labelled mesh (mesh_utilities.py:28-48).

    Every sphere has radius ``threshold_dist`` x (smallest nonzero distance between
    the points) / 2 and is an icosahedron subdivided ``n_subdivisions`` times with
    its vertices pushed to the sphere; sphere ``i`` gets face labels (0, i + 1).
    Returns ``(verts[nv, 3] float64, faces[nt, 5] int32)`` as
    ``combine_all_verts_faces_mm`` assembles them.  The reference takes trimesh's
    primitive sphere, the same construction; this library's icosphere lists the
    vertices and faces in its own order (the same points, faces outward).  Fewer
    than two distinct points raise ``ValueError`` (the smallest distance is
    undefined), as in the reference.
    """
    from scipy.spatial.distance import cdist

    from .mesh import icosphere

    points = np.asarray(points, dtype=np.float64)
    d = cdist(points, points)
    min_dist = np.amin(d[d != 0]) * threshold_dist
    all_verts, all_faces = [], []
    for i in range(len(points)):
        v, f = icosphere(int(n_subdivisions), radius=min_dist / 2, center=points[i])
        labels = np.stack([np.zeros(len(f)), np.full(len(f), float(i + 1))], axis=1)
        all_verts.append(v)
        all_faces.append(np.concatenate([f.astype(np.float64), labels], axis=1))
    return combine_all_verts_faces_mm(all_verts, all_faces)

