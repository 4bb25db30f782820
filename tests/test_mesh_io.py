"""Mesh files (.obj, .rec) and the reference's mesh assembly helpers
(deltamic/mesh_utilities.py:8-25)."""
import os

import numpy as np
import pytest

from deltamic_b200.mesh import icosphere
from deltamic_b200.mesh_io import (combine_all_verts_faces, combine_all_verts_faces_mm, read_obj,
                                   read_rec, write_obj, write_rec)

# mesh files shipped with the reference (data/mesh), when $DELTAMIC_REF names a checkout
REF_DATA = os.path.join(os.environ.get("DELTAMIC_REF", ""), "data", "mesh")


def test_obj_round_trip_and_face_forms(tmp_path):
    v, f = icosphere(2, 0.3)
    p = tmp_path / "s.obj"
    write_obj(p, v, f)
    v2, f2 = read_obj(p)
    assert np.array_equal(v2, v) and np.array_equal(f2, f)
    q = tmp_path / "q.obj"
    q.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 0 0 0\n"
                 "vt 0 0\nf 1/1 2/1 3/1 4/1\nf -5//1 -4//1 -1//1\n")
    vq, fq = read_obj(q, merge=False)
    assert vq.shape == (5, 3) and fq.tolist() == [[0, 1, 2], [0, 2, 3], [0, 1, 4]]
    vm, fm = read_obj(q)                 # vertex 4 duplicates vertex 0
    assert vm.shape == (4, 3) and fm.tolist() == [[0, 1, 2], [0, 2, 3], [0, 1, 0]]


def test_rec_round_trip(tmp_path):
    v1, f1 = icosphere(1, 0.2)
    v2, f2 = icosphere(1, 0.2, center=(0.5, 0, 0))
    mm = [np.hstack([f1, np.full((len(f1), 1), 1), np.zeros((len(f1), 1), int)]),
          np.hstack([f2, np.full((len(f2), 1), 2), np.zeros((len(f2), 1), int)])]
    V, F = combine_all_verts_faces_mm([v1, v2], mm)
    assert F.dtype == np.int32 and F[len(f1):, :3].min() == len(v1)
    p = tmp_path / "two.rec"
    write_rec(p, V, F)
    Vr, Fr = read_rec(p)
    assert np.array_equal(Vr, V) and np.array_equal(Fr, F)
    Vc, Fc = combine_all_verts_faces([v1, v2], [f1.copy(), f2.copy()])
    assert np.array_equal(Fc[len(f1):], f2 + len(v1))


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="$DELTAMIC_REF not set to a reference checkout")
def test_reference_data_files_read():
    for name, nv, nt in (("cow.obj", 2930, 5856), ("fish.obj", 7106, 14208)):
        v, f = read_obj(os.path.join(REF_DATA, name))
        assert v.shape == (nv, 3) and f.shape == (nt, 3)
    v, f = read_rec(os.path.join(REF_DATA, "Sample01_007.rec"))
    assert v.shape == (1996, 3) and f.shape == (4055, 5)
    assert set(np.unique(f[:, 3:]).tolist()) == {0, 1, 2, 3}


def test_create_initial_mesh_from_points_mm():
    """mesh_utilities.py:28-48: radius = threshold * (smallest pairwise distance) / 2,
    one sphere of 10*4^n + 2 vertices / 20*4^n faces per point, labels (0, i + 1),
    faces offset per sphere, int32; every face outward and every vertex on its
    sphere."""
    from scipy.spatial.distance import cdist

    from deltamic_b200 import create_initial_mesh_from_points_mm
    pts = np.array([[0.0, 0.0, 0.0], [1.0, 0.2, 0.0], [0.3, 1.5, -0.4]])
    n = 2
    V, F = create_initial_mesh_from_points_mm(pts, n_subdivisions=n, threshold_dist=0.9)
    nv1, nf1 = 10 * 4 ** n + 2, 20 * 4 ** n
    assert V.shape == (3 * nv1, 3) and V.dtype == np.float64
    assert F.shape == (3 * nf1, 5) and F.dtype == np.int32
    d = cdist(pts, pts)
    radius = d[d != 0].min() * 0.9 / 2
    for i in range(3):
        vi = V[i * nv1:(i + 1) * nv1]
        fi = F[i * nf1:(i + 1) * nf1]
        assert np.allclose(np.linalg.norm(vi - pts[i], axis=1), radius, rtol=1e-12)
        assert (fi[:, 3] == 0).all() and (fi[:, 4] == i + 1).all()
        assert fi[:, :3].min() == i * nv1 and fi[:, :3].max() == (i + 1) * nv1 - 1
        t = V[fi[:, :3]]
        nrm = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
        assert (np.einsum("ij,ij->i", nrm, t.mean(axis=1) - pts[i]) > 0).all()
    with pytest.raises(ValueError):
        create_initial_mesh_from_points_mm(pts[:1])
