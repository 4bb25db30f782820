"""The kernel's per-pair math (pair_math.cuh) compiled for the host with g++ and
checked against the oracle's F and dF/dx (the device build differs only in using
the MUFU sin/cos/rcp approximations)."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT, load_golden
from deltamic_b200.mesh import icosphere, sh_perturb


@pytest.fixture(scope="module")
def hostlib(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("hostpair") / "libhostpair.so")
    src = os.path.join(ROOT, "tests", "host_pairmath.cpp")
    subprocess.run([gxx, "-O2", "-shared", "-fPIC", "-std=c++17", "-o", out, src], check=True)
    return ctypes.CDLL(out)


def _run(lib, v, f, m, lo, L, fast):
    n, nt = len(m), len(f)
    F = np.zeros((n, nt, 2), np.float32)
    dF = np.zeros((n, nt, 3, 2), np.float32)
    sp = np.zeros((n, nt), np.uint8)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    vv = np.ascontiguousarray(v, np.float64)
    ff = np.ascontiguousarray(f, np.int64)
    mm = np.ascontiguousarray(m, np.int32)
    lo = np.ascontiguousarray(lo, np.float64)
    L = np.ascontiguousarray(L, np.float64)
    lib.dm_host_pairs(P(vv), P(ff), ctypes.c_int64(nt), P(mm), ctypes.c_int64(n), P(lo), P(L),
                      P(F), P(dF), P(sp), ctypes.c_int(fast))
    return F[..., 0] + 1j * F[..., 1], dF[..., 0] + 1j * dF[..., 1], sp


def _reference(v, f, m, box, shape):
    axes = oracle.frequency_axes(box, shape)
    k = (m + (np.array(shape) - 1)) // 2
    xi = np.stack([axes[d][k[:, d]] for d in range(3)], 1)
    xiv = xi @ (v - box[:, 0]).T
    return oracle.pair_F_and_grads(xiv[:, f[:, 0]], xiv[:, f[:, 1]], xiv[:, f[:, 2]])


@pytest.mark.parametrize("shape", [(21, 21, 21), (64, 64, 64)])
@pytest.mark.parametrize("fast", [1, 0])
def test_pair_math_matches_oracle(hostlib, shape, fast):
    rng = np.random.default_rng(0)
    v, f = icosphere(2, 0.3)
    v, _ = sh_perturb(v, 4, 0.08, rng, radius=0.3)
    box = oracle.compute_box_size(v, 0.2)
    k = np.stack([rng.integers(0, s, 1500) for s in shape], 1)
    m = (2 * k - (np.array(shape) - 1)).astype(np.int32)
    F, dF, sp = _run(hostlib, v, f, m, box[:, 0], box[:, 1] - box[:, 0], fast)
    F0, g0 = _reference(v, f, m, box, shape)
    assert np.linalg.norm(F - F0) / np.linalg.norm(F0) < 2e-6
    for i in range(3):
        assert np.linalg.norm(dF[..., i] - g0[i]) / np.linalg.norm(g0[i]) < 2e-6
    assert 0 < sp.mean() < 0.2


def test_pair_math_degenerate_branches(hostlib):
    """Axis-aligned faces on an odd grid: exact zeros in the phase differences."""
    d = load_golden("cube_degenerate")
    box, shape = d["box_size"], tuple(int(s) for s in d["box_shape"])
    axes_k = np.stack(np.unravel_index(d["idx"], shape), 1)
    m = (2 * axes_k - (np.array(shape) - 1)).astype(np.int32)
    F, dF, sp = _run(hostlib, d["verts"], d["faces"], m, box[:, 0], box[:, 1] - box[:, 0], 1)
    F0, g0 = _reference(d["verts"], d["faces"], m, box, shape)
    assert sp.mean() > 0.01
    assert np.max(np.abs(F - F0)) < 2e-6
    for i in range(3):
        assert np.max(np.abs(dF[..., i] - g0[i])) < 1e-5 * max(1.0, np.abs(g0[i]).max())
