"""Oracle of the surface + enclosed-volume ("autofluorescence") transform
(deltamic/render.py:228-318) against golden vectors made by the reference
function itself (tests/golden/make_golden_volume.py), plus its known answers."""
import numpy as np
import torch

import oracle.volume as ov
from conftest import band_xi, rel_l2
from deltamic_b200 import (compute_volume_manifold, get_internal_triangle_and_mesh_areas,
                           get_internal_triangle_and_mesh_areas_and_normals)
from deltamic_b200.mesh import icosphere, random_sh_shape


def test_oracle_volume_matches_reference(golden_volume):
    name, g = golden_volume
    xi = band_xi(g["box_shape"], g["lengths"], g["idx"])
    ft, _ = ov.volume_forward(g["verts"], g["faces"], float(g["regint"]), xi)
    ref = g["ft"]
    live = ~np.isnan(ref)
    assert rel_l2(ft[live], ref[live]) < 1e-12
    if not live.all():  # xi = 0 on an odd grid: 0/0 in the reference, the limit here
        assert int((~live).sum()) == 1
        assert abs(ft[~live][0] - (1.0 - float(g["regint"]))) < 1e-12
    if "w" in g:
        gv, gr = ov.volume_backward(g["verts"], g["faces"], float(g["regint"]), xi, g["w"])
        assert rel_l2(gv, g["grad_verts"]) < 1e-8
        assert abs(gr - float(g["grad_regint"])) < 1e-9 * max(1.0, abs(gr))


def test_volume_term_is_the_enclosed_ball_transform():
    """For a fine sphere the volume part per unit beta tends to the transform of
    the ball, 4 pi (sin kR - kR cos kR) / k^3, and the value at xi -> 0 to
    1 - regint."""
    v, f = icosphere(4, 0.3)
    xi = np.array([[5.0, 0, 0], [0, 10.0, 0], [7.0, 7.0, 7.0], [1e-3, 2e-3, -1e-3]])
    ft, vol = ov.volume_forward(v, f, 0.6, xi)
    k = np.linalg.norm(xi, axis=1)
    R = 0.3
    ball = 4 * np.pi * (np.sin(k * R) - k * R * np.cos(k * R)) / k ** 3
    assert np.max(np.abs(vol.real / ball - 1.0)) < 3e-3
    assert np.max(np.abs(vol.imag)) < 1e-9
    assert abs(ft[3] - 0.4) < 1e-5


def test_torch_helpers_match_oracle_geometry():
    """The plain-torch helpers of the reference API (render.py:184-226)."""
    v, f = random_sh_shape(2, 0.3, 4, 0.08, seed=3)
    V, F = torch.tensor(v, dtype=torch.float64), torch.tensor(f)
    area, total, nor = get_internal_triangle_and_mesh_areas_and_normals(V, F)
    a2, t2 = get_internal_triangle_and_mesh_areas(V, F)
    _, a64, n64, rv64 = ov._geometry(v, f)
    assert rel_l2(area.numpy(), a64) < 1e-12 and rel_l2(a2.numpy(), a64) < 1e-12
    assert abs(float(total) - a64.sum()) < 1e-12 and abs(float(t2) - a64.sum()) < 1e-12
    assert rel_l2(nor.numpy(), n64) < 1e-12
    assert abs(float(compute_volume_manifold(V, F)) - rv64) < 1e-12 * abs(rv64)
