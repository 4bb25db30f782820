"""The C-ABI library: builds, loads without a GPU, exports every declared symbol,
and rejects bad arguments on the host before touching the device."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "deltamic_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dm_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from deltamic_b200 import _native
    if not os.path.exists(_native.LIB_PATH):
        from deltamic_b200 import build
        build.build()
    return _native.lib()


def test_every_declared_symbol_is_exported_and_bound(lib):
    from deltamic_b200 import _native
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
        assert n in _native.SIGNATURES, n
    assert set(_native.SIGNATURES) == set(names)


def test_abi_version_and_status_strings(lib):
    assert lib.dm_abi_version() == 2
    assert lib.dm_status_string(0) == b"ok"
    assert b"index" in lib.dm_status_string(2)


def test_host_side_argument_checks(lib):
    from deltamic_b200 import _native as N
    box = N.make_box([[0, 1], [0, 1], [0, 1]], (8, 8, 8))
    bad = N.make_box([[0, 1], [0, 1], [1, 0]], (8, 8, 8))
    # null workspace / bad box / negative sizes: rejected before any launch
    assert lib.dm_meshft_forward(None, 3, None, 1, None, ctypes.byref(box), None, 0, None, None,
                                 None, None, 0, None) & N.DM_ERR_INVALID_ARG
    assert lib.dm_meshft_forward(None, 0, None, 0, None, ctypes.byref(bad), None, 0, None, None,
                                 None, ctypes.c_void_p(16), 1 << 20, None) == N.DM_ERR_INVALID_ARG
    assert lib.dm_meshft_backward(None, -1, None, 0, None, ctypes.byref(box), None, 0, None, None,
                                  None, 1.0, None, None, None, None, None, None, 0,
                                  None) == N.DM_ERR_SIZE
    assert lib.dm_image_loss(None, 10, 0, None, 0.0, None, None, None, None, 0,
                             None) == N.DM_ERR_INVALID_ARG
    assert lib.dm_narrowband_compact(None, -1, 0.0, None, None, None, 0,
                                     None) == N.DM_ERR_INVALID_ARG
    # workspace smaller than the query
    need = lib.dm_meshft_forward_workspace_size(10, 16, 100)
    assert need > 0
    assert lib.dm_meshft_forward(ctypes.c_void_p(16), 10, ctypes.c_void_p(16), 16,
                                 ctypes.c_void_p(16), ctypes.byref(box), ctypes.c_void_p(16),
                                 100, None, ctypes.c_void_p(16), None, ctypes.c_void_p(16),
                                 need - 1, None) == N.DM_ERR_WORKSPACE


def test_workspace_sizes_grow_with_problem(lib):
    a = lib.dm_meshft_backward_workspace_size(642, 1280, 24464)
    b = lib.dm_meshft_backward_workspace_size(10242, 20480, 14064)
    assert 0 < a < b
    assert lib.dm_topology_size(10242, 20480) > 4 * 3 * 20480


def test_product_path_refuses_cpu():
    import torch
    import deltamic_b200 as dm
    with pytest.raises(RuntimeError):
        dm.Fourier3dMesh(torch.tensor([[0.0, 1.0]] * 3), (8, 8, 8), device="cpu")


def test_bandbox_render_host_checks(lib):
    """Band boxes the line kernels do not serve are refused before any launch."""
    from deltamic_b200 import _native as N
    box = N.make_box([[0, 1], [0, 1], [0, 1]], (64, 64, 128))
    wide = (ctypes.c_int32 * 6)(0, 0, 0, 63, 63, 64)  # axis-2 extent 65 > 64
    narrow = (ctypes.c_int32 * 6)(10, 12, 20, 50, 52, 41)
    outside = (ctypes.c_int32 * 6)(10, 12, 20, 50, 64, 41)
    two_chunks = (ctypes.c_int32 * 6)(10, 12, 20, 50, 52, 83)  # extent 64: served
    assert lib.dm_render_loss_bandbox_supported(ctypes.byref(box), two_chunks) == 1
    assert lib.dm_render_loss_bandbox_supported(ctypes.byref(box), wide) == 0
    assert lib.dm_render_loss_bandbox_supported(ctypes.byref(box), narrow) == 1
    assert lib.dm_render_loss_bandbox_supported(ctypes.byref(box), outside) == 0
    assert lib.dm_render_loss_bandbox_workspace_size(ctypes.byref(box), narrow) > 64 ** 3 * 16
    fake = ctypes.c_void_p(16)
    st = lib.dm_render_loss_bandbox(fake, fake, 1, ctypes.byref(box), wide, None, 0, None, 0.0,
                                    fake, None, None, fake, 1 << 30, None)
    assert st == N.DM_ERR_UNSUPPORTED
    # mse without a target, and a workspace below the query
    assert lib.dm_render_loss_bandbox(fake, fake, 1, ctypes.byref(box), narrow, None, 1, None,
                                      0.0, fake, None, None, fake, 1 << 30,
                                      None) == N.DM_ERR_INVALID_ARG
    assert lib.dm_render_loss_bandbox(fake, fake, 1, ctypes.byref(box), narrow, None, 0, None,
                                      0.0, fake, None, None, fake, 1024,
                                      None) == N.DM_ERR_WORKSPACE


def test_conv_host_checks(lib):
    """Convolution entry points: shapes outside the kernels' limits (Co not in
    {16, 32, 64, 128}, Ci > 128, tensors of 2^31 elements or more) are refused on the
    host; the workspace holds dP (BF16) and the weight-gradient split partials with
    the bias row."""
    from deltamic_b200 import _native as N
    assert lib.dm_conv3d_s2_workspace_size(2, 16, 16, 16, 1, 24) == 0
    assert lib.dm_conv3d_s2_workspace_size(2, 16, 16, 16, 129, 32) == 0
    assert lib.dm_conv3d_s2_workspace_size(1024, 128, 128, 128, 1, 16) == 0  # 2^31 * 16
    ws = lib.dm_conv3d_s2_workspace_size(2, 16, 16, 16, 16, 32)
    M, Kp = 2 * 8 ** 3, 448
    assert ws >= M * 32 * 2 + (Kp + 1) * 32 * 4
    assert lib.dm_conv3d_s2_forward(None, 2, 16, 16, 16, 16, None, None, 32, None, None,
                                    None) == N.DM_ERR_INVALID_ARG
    assert lib.dm_conv3d_s2_forward(ctypes.c_void_p(16), 2, 16, 16, 16, 16, ctypes.c_void_p(16),
                                    None, 48, ctypes.c_void_p(16), ctypes.c_void_p(16),
                                    None) == N.DM_ERR_INVALID_ARG
    p = ctypes.c_void_p(16)
    assert lib.dm_conv3d_s2_backward(p, 2, 16, 16, 16, 16, p, 32, p, p, None, p, p, p, ws - 1,
                                     None) == N.DM_ERR_WORKSPACE
    assert lib.dm_conv3d_s2_device_error(None, None) == N.DM_ERR_INVALID_ARG


def test_header_and_library_from_plain_c(lib, tmp_path):
    """A C99 program (tests/abi_host_check.c) compiles against the public header
    with -Wall -Wextra -pedantic -Werror, links the shared library and runs its
    host-side calls: the boundary is usable from C, not only through ctypes."""
    import shutil
    import subprocess
    from deltamic_b200 import _native
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    libdir = os.path.dirname(_native.LIB_PATH)
    exe = str(tmp_path / "abi_host_check")
    subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                    "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "abi_host_check.c"),
                    "-L", libdir, "-ldeltamic_b200", f"-Wl,-rpath,{libdir}", "-o", exe],
                   check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "ok"
