"""The allocation-free meshFT forward (dm_meshft_forward_noalloc).

Some callers may not allocate device memory when they render: their host
framework owns every device byte, or they allocate only at start-up.  For them
the library keeps a fixed 8 MiB scratch array of its own.  This test calls that
entry point through the C ABI twice in a row and checks each result against the
regular dm_meshft_forward (which uses a caller-provided workspace) and against
the float64 oracle, reads the fixed scratch's status word after each call,
checks that a face index out of range is reported through that word, and that
a request too large for the fixed scratch is refused before any launch.
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


def _case():
    v, f = random_sh_shape(3, 0.3, 4, 0.08, seed=21)
    rng = np.random.default_rng(21)
    c = rng.uniform(0.5, 1.5, len(f))
    box = oracle.compute_box_size(v, 0.2)
    shape = (48, 44, 40)
    grid = ops.FreqGrid(box, shape)
    xi = grid.axes(torch.float32, DEV)
    otf = ops.gaussian_otf(torch.diag(torch.tensor([1e-3, 1e-3, 4e-3], device=DEV)), *xi)
    band = ops.narrowband(otf, 1e-5)
    return v, f, c, box, shape, grid, otf, band


def _status(lib):
    flags = N._INT()
    N.check(lib.dm_meshft_forward_noalloc_device_error(ctypes.byref(flags), N.stream_ptr(DEV)),
            "dm_meshft_forward_noalloc_device_error")
    return flags.value


def _call(lib, V, F, C, grid, band, otf, out, out_grid):
    return lib.dm_meshft_forward_noalloc(
        N.ptr(V), V.shape[0], N.ptr(F), F.shape[0], N.ptr(C), ctypes.byref(grid.cbox),
        N.ptr(band), band.numel(), N.ptr(otf), N.ptr(out),
        N.ptr(out_grid) if out_grid is not None else None, N.stream_ptr(DEV))


def test_noalloc_forward_matches_workspace_forward_and_oracle_twice():
    lib = N.lib()
    v, f, c, box, shape, grid, otf, band = _case()
    V = torch.tensor(v, dtype=torch.float32, device=DEV)
    F = torch.tensor(f, device=DEV)
    C = torch.tensor(c, dtype=torch.float32, device=DEV)
    nv, nt, nb = V.shape[0], F.shape[0], band.numel()
    assert lib.dm_meshft_forward_workspace_size(nv, nt, nb) <= 8 << 20

    ref_grid = torch.zeros(shape, dtype=torch.complex64, device=DEV)
    ref = ops.meshft_list(V, F, C, grid, band, otf=otf, spectrum=ref_grid)
    axes = oracle.frequency_axes(box, shape)
    xil = oracle.xi_list_from_band(band.cpu().numpy().astype(np.int64), axes)
    ft64 = oracle.meshft_forward(v - box[:, 0], f, c, xil)
    for _ in range(2):
        out = torch.full((nb,), float("nan"), dtype=torch.complex64, device=DEV)
        out_grid = torch.zeros(shape, dtype=torch.complex64, device=DEV)
        N.check(_call(lib, V, F, C, grid, band, otf, out, out_grid), "dm_meshft_forward_noalloc")
        torch.cuda.synchronize()
        assert _status(lib) == 0
        got = out.cpu().numpy()
        assert rel_l2(got, ref.cpu().numpy()) < TOL_FT
        assert rel_l2(out_grid.cpu().numpy(), ref_grid.cpu().numpy()) < TOL_FT
        assert rel_l2(got, ft64) < TOL_FT


def test_noalloc_forward_reports_bad_face_index():
    """A face index past the vertex count (made on the host) is clamped by the
    face-record kernel and reported in the fixed scratch's status word; the next
    good call starts from a cleared word."""
    lib = N.lib()
    v, f, c, box, shape, grid, otf, band = _case()
    V = torch.tensor(v, dtype=torch.float32, device=DEV)
    C = torch.tensor(c, dtype=torch.float32, device=DEV)
    bad = np.array(f, copy=True)
    bad[7, 1] = len(v) + 5
    out = torch.empty(band.numel(), dtype=torch.complex64, device=DEV)
    st = _call(lib, V, torch.tensor(bad, device=DEV), C, grid, band, otf, out, None)
    assert st == N.DM_OK
    assert _status(lib) & N.DM_ERR_BAD_INDEX
    assert _status(lib) == 0  # cleared by the read
    N.check(_call(lib, V, torch.tensor(f, device=DEV), C, grid, band, otf, out, None),
            "dm_meshft_forward_noalloc")
    assert _status(lib) == 0


def test_noalloc_forward_rejects_oversize_and_bad_args_before_launch():
    lib = N.lib()
    box = N.make_box([[0, 1], [0, 1], [0, 1]], (256, 256, 256))
    # a band far larger than the fixed scratch can hold partial sums for
    st = lib.dm_meshft_forward_noalloc(None, 10, None, 200000, None, ctypes.byref(box), None,
                                       5_000_000, None, None, None, None)
    assert st == N.DM_ERR_SIZE
    # null mesh pointers with faces present: refused on the host
    st = lib.dm_meshft_forward_noalloc(None, 10, None, 16, None, ctypes.byref(box), None,
                                       0, None, None, None, None)
    assert st == N.DM_ERR_INVALID_ARG
    assert lib.dm_meshft_forward_noalloc(None, 0, None, 0, None, None, None, 0, None, None,
                                         None, None) == N.DM_ERR_INVALID_ARG
