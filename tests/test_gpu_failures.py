"""Failure detection on the device, without faulting the GPU: a bounded wait that
runs out ends its kernel with DM_ERR_TIMEOUT in a status word (the context stays
usable), and non-finite vertex coordinates are reported as DM_ERR_NONFINITE
instead of reaching the fixed-point conversion."""
import ctypes

import numpy as np
import pytest
import torch

import oracle
from deltamic_b200 import _native as N
from deltamic_b200 import ops
from deltamic_b200.mesh import random_sh_shape

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.mark.parametrize("mode,limit", [(0, 1 << 14), (1, 40)])
def test_bounded_wait_runs_out_with_timeout_status(mode, limit):
    lib = N.lib()
    st = torch.zeros(1, dtype=torch.int32, device=DEV)
    N.check(lib.dm_selftest_bounded_wait(mode, limit, N.ptr(st), N.stream_ptr(DEV)),
            "dm_selftest_bounded_wait")
    torch.cuda.synchronize()
    assert int(st.item()) == N.DM_ERR_TIMEOUT
    # the context is usable afterwards: a regular launch runs and is correct
    x = torch.arange(10, device=DEV, dtype=torch.float32)
    assert float((x * 2).sum()) == 90.0
    assert lib.dm_selftest_bounded_wait(mode, 0, N.ptr(st), N.stream_ptr(DEV)) == \
        N.DM_ERR_INVALID_ARG
    assert lib.dm_selftest_bounded_wait(0, (1 << 22) + 1, N.ptr(st), N.stream_ptr(DEV)) == \
        N.DM_ERR_SIZE


@pytest.mark.parametrize("bad", [float("nan"), float("inf")])
def test_nonfinite_vertex_reported_in_status_word(bad):
    lib = N.lib()
    v, f = random_sh_shape(2, 0.3, 4, 0.08, seed=3)
    v = v.copy()
    v[17, 1] = bad
    box = oracle.compute_box_size(np.nan_to_num(v, nan=0.0, posinf=0.0), 0.2)
    grid = ops.FreqGrid(box, (16, 16, 16))
    xi = grid.axes(torch.float32, DEV)
    otf = ops.gaussian_otf(torch.eye(3, device=DEV) * 1e-3, *xi)
    band = ops.narrowband(otf, 1e-5)
    V = torch.tensor(v, dtype=torch.float32, device=DEV)
    F = torch.tensor(f, device=DEV)
    C = torch.ones(len(f), device=DEV)
    nb = band.numel()
    ws = torch.zeros(lib.dm_meshft_forward_workspace_size(len(v), len(f), nb),
                     dtype=torch.uint8, device=DEV)
    ft = torch.empty(nb, dtype=torch.complex64, device=DEV)
    st = lib.dm_meshft_forward(N.ptr(V), len(v), N.ptr(F), len(f), N.ptr(C),
                               ctypes.byref(grid.cbox), N.ptr(band), nb, None, N.ptr(ft), None,
                               N.ptr(ws), ws.numel(), N.stream_ptr(DEV))
    assert st == N.DM_OK
    flags = N._INT()
    assert lib.dm_device_error(N.ptr(ws), ctypes.byref(flags), N.stream_ptr(DEV)) == N.DM_OK
    assert flags.value & N.DM_ERR_NONFINITE
    # the explicit-list path reports it as well (its cell sizing skips the value)
    X = torch.tensor(np.random.default_rng(0).normal(size=(50, 3)) * 20, dtype=torch.float32,
                     device=DEV)
    wsx = torch.zeros(lib.dm_meshft_forward_xi_workspace_size(len(v), len(f), 50),
                      dtype=torch.uint8, device=DEV)
    ftx = torch.empty(50, dtype=torch.complex64, device=DEV)
    assert lib.dm_meshft_forward_xi(N.ptr(V), len(v), N.ptr(F), len(f), N.ptr(C), N.ptr(X), 50,
                                    N.ptr(ftx), N.ptr(wsx), wsx.numel(),
                                    N.stream_ptr(DEV)) == N.DM_OK
    assert lib.dm_device_error(N.ptr(wsx), ctypes.byref(flags), N.stream_ptr(DEV)) == N.DM_OK
    assert flags.value & N.DM_ERR_NONFINITE
