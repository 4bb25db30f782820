"""The allocation-free meshFT forward (dm_meshft_forward_noalloc).

Some callers may not allocate device memory when they render: their host
framework owns every device byte, or they allocate only at start-up.  For them
the library keeps a fixed 8 MiB scratch array of its own.  This test calls that
entry point through the C ABI twice in a row and checks each result against the
regular dm_meshft_forward (which uses a caller-provided workspace), and checks
that a request too large for the fixed scratch is refused before any launch.
The file is named to be collected last."""
import ctypes

import numpy as np
import pytest
import torch

import oracle
from conftest import rel_l2
from deltamic_b200 import _native as N
from deltamic_b200 import ops
from deltamic_b200.mesh import random_sh_shape

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL_FT = 1e-5  # the forward tolerance of the other GPU tests


def test_noalloc_forward_matches_workspace_forward_twice():
    lib = N.lib()
    v, f = random_sh_shape(3, 0.3, 4, 0.08, seed=21)
    rng = np.random.default_rng(21)
    c = rng.uniform(0.5, 1.5, len(f))
    box = oracle.compute_box_size(v, 0.2)
    shape = (48, 44, 40)
    grid = ops.FreqGrid(box, shape)
    xi = grid.axes(torch.float32, DEV)
    otf = ops.gaussian_otf(torch.diag(torch.tensor([1e-3, 1e-3, 4e-3], device=DEV)), *xi)
    band = ops.narrowband(otf, 1e-5)
    V = torch.tensor(v, dtype=torch.float32, device=DEV)
    F = torch.tensor(f, device=DEV)
    C = torch.tensor(c, dtype=torch.float32, device=DEV)
    nv, nt, nb = V.shape[0], F.shape[0], band.numel()
    assert lib.dm_meshft_forward_workspace_size(nv, nt, nb) <= 8 << 20

    ref_grid = torch.zeros(shape, dtype=torch.complex64, device=DEV)
    ref = ops.meshft_list(V, F, C, grid, band, otf=otf, spectrum=ref_grid)
    for _ in range(2):
        out = torch.full((nb,), float("nan"), dtype=torch.complex64, device=DEV)
        out_grid = torch.zeros(shape, dtype=torch.complex64, device=DEV)
        st = lib.dm_meshft_forward_noalloc(
            N.ptr(V), nv, N.ptr(F), nt, N.ptr(C), ctypes.byref(grid.cbox), N.ptr(band), nb,
            N.ptr(otf), N.ptr(out), N.ptr(out_grid), N.stream_ptr(DEV))
        N.check(st, "dm_meshft_forward_noalloc")
        torch.cuda.synchronize()
        assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) < TOL_FT
        assert rel_l2(out_grid.cpu().numpy(), ref_grid.cpu().numpy()) < TOL_FT


def test_noalloc_forward_rejects_oversize_before_launch():
    lib = N.lib()
    box = N.make_box([[0, 1], [0, 1], [0, 1]], (256, 256, 256))
    # a band far larger than the fixed scratch can hold partial sums for
    st = lib.dm_meshft_forward_noalloc(None, 10, None, 200000, None, ctypes.byref(box), None,
                                       5_000_000, None, None, None, None)
    assert st == N.DM_ERR_SIZE
