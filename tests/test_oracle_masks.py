"""Oracle of the segmentation masks (deltamic/mask_creation.py): known answers.
The reference's mask functions need trimesh, absent here, so the oracle is checked
against properties of the masks rather than against reference outputs."""
import numpy as np

import oracle.masks as om
from deltamic_b200.mesh import icosphere


def _box(v, pad=0.15):
    lo, hi = v.min(0) - pad, v.max(0) + pad
    return np.stack([lo, hi], axis=1)


def test_membrane_points_are_on_the_sphere_shell():
    v, f = icosphere(2, 0.3)
    shape = (20, 20, 20)
    box = _box(v)
    m = om.semantic_mask(v, f, shape, box)
    pts = om.create_coords(shape, box)[m == 1]
    r = np.linalg.norm(pts, axis=1)
    h = (box[0, 1] - box[0, 0]) / 19
    assert len(pts) > 100 and np.all(np.abs(r - 0.3) < h)


def test_instance_mask_labels_inside_and_outside():
    v, f = icosphere(2, 0.3)
    faces = np.hstack([f, np.ones((len(f), 1), int), np.zeros((len(f), 1), int)])
    shape = (16, 16, 16)
    box = _box(v)
    lab = om.instance_mask(v, faces, shape, box)
    pts = om.create_coords(shape, box).reshape(*shape, 3)
    r = np.linalg.norm(pts, axis=3)
    assert np.all(lab[r < 0.25] == 2) and np.all(lab[r > 0.35] == 1)
