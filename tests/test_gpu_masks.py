"""Segmentation masks on the GPU against the oracle's restatement of
deltamic/mask_creation.py (trimesh's refinement and scipy's KDTree): integer
results, compared exactly (the meshes are jittered so no grid point is equidistant
from two samples)."""
import numpy as np
import pytest

import oracle.masks as om
from deltamic_b200 import create_instance_segmentation_mask, create_semantic_segmentation_mask
from deltamic_b200.mesh import icosphere, jitter, random_sh_shape
from deltamic_b200.mesh_io import combine_all_verts_faces_mm

pytestmark = pytest.mark.gpu


def _box(v, pad=0.15):
    return np.stack([v.min(0) - pad, v.max(0) + pad], axis=1)


@pytest.mark.parametrize("level,shape", [(1, (24, 24, 24)), (2, (20, 18, 16)), (3, (40, 36, 33))])
def test_membrane_mask_matches_oracle(level, shape):
    v, f = random_sh_shape(level, 0.3, 4, 0.08, seed=level)
    v = jitter(v, 1e-3, np.random.default_rng(level))
    box = _box(v)
    got = create_semantic_segmentation_mask(v, f, np.array(shape), box)
    ref = om.semantic_mask(v, f, np.array(shape), box)
    assert got.shape == ref.shape == (int(np.prod(shape)),)
    print(f"level {level} {shape}: {int(ref.sum())} membrane voxels, "
          f"{int((got != ref).sum())} differ")
    assert np.array_equal(got, ref)


def _two_cells():
    rng = np.random.default_rng(5)
    v1, f1 = icosphere(2, 0.25)
    v2, f2 = icosphere(2, 0.2, center=(0.5, 0.05, 0.0))
    v1, v2 = jitter(v1, 2e-3, rng), jitter(v2, 2e-3, rng)
    # cell 1: labels (1, 0); cell 2 stored with the smaller label first, so it is
    # flipped by reorder_faces
    mm = [np.hstack([f1, np.full((len(f1), 1), 1), np.zeros((len(f1), 1), int)]),
          np.hstack([f2[:, [0, 2, 1]], np.zeros((len(f2), 1), int), np.full((len(f2), 1), 2)])]
    return combine_all_verts_faces_mm([v1, v2], mm)


@pytest.mark.parametrize("shape", [(12, 10, 9), (24, 20, 18), (64, 48, 48), (96, 80, 72)])
def test_instance_mask_matches_oracle(shape):
    V, F = _two_cells()
    box = _box(V, 0.1)
    got = create_instance_segmentation_mask(V, F.astype(np.int64), np.array(shape), box)
    ref = om.instance_mask(V, F.astype(np.int64), np.array(shape), box)
    assert got.shape == ref.shape == shape
    print(f"{shape}: labels {np.unique(ref).tolist()}, {int((got != ref).sum())} differ")
    assert np.array_equal(got, ref)
