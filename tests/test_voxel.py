"""Occupancy for the IoU of fits: the parity rule (oracle restatement of the
kernel) against the winding number, and the CUDA voxelizer against the oracle."""
import numpy as np
import pytest
import torch

import oracle
from oracle.voxel import occupancy_parity, occupancy_winding
from deltamic_b200.mesh import icosphere, random_sh_shape


def test_parity_equals_winding_number():
    v, f = random_sh_shape(2, 0.3, 4, 0.08, seed=5)
    box = oracle.compute_box_size(v, 0.3)
    a = occupancy_parity(v, f, box, (20, 18, 22))
    b = occupancy_winding(v, f, box, (20, 18, 22))
    assert (a != b).sum() == 0
    assert 0.1 < a.mean() < 0.9


def test_sphere_volume_fraction():
    v, f = icosphere(4, 0.3)
    box = np.array([[-0.5, 0.5]] * 3)
    a = occupancy_parity(v, f, box, (40, 40, 40))
    frac = a.mean()
    assert abs(frac - 4 / 3 * np.pi * 0.3 ** 3) < 0.01


@pytest.mark.gpu
def test_cuda_voxelizer_matches_oracle():
    from deltamic_b200 import ops
    v, f = random_sh_shape(3, 0.3, 6, 0.08, seed=8)
    box = oracle.compute_box_size(v, 0.2)
    shape = (32, 30, 28)
    grid = ops.FreqGrid(box, shape)
    V = torch.tensor(v, dtype=torch.float32, device="cuda:0")
    F = torch.tensor(f, device="cuda:0")
    occ = ops.voxelize(V, F, grid).cpu().numpy()
    ref = occupancy_parity(V.cpu().double().numpy(), f, box, shape)
    assert (occ != ref).sum() <= 2  # float32 vertices, double crossings: ties only
    assert ops.iou(torch.tensor(occ), torch.tensor(ref)) > 0.999
