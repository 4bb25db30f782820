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


def _run(lib, v, f, m, g, lo, L):
    n, nt = len(m), len(f)
    F = np.zeros((n, nt, 2), np.float32)
    z = np.zeros((n, nt, 3), np.float32)
    r = np.zeros((n, nt), np.float32)
    cls = np.zeros((n, nt), np.uint8)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    vv = np.ascontiguousarray(v, np.float64)
    ff = np.ascontiguousarray(f, np.int64)
    mm = np.ascontiguousarray(m, np.int32)
    gg = np.ascontiguousarray(np.stack([g.real, g.imag], 1), np.float32)
    lo = np.ascontiguousarray(lo, np.float64)
    L = np.ascontiguousarray(L, np.float64)
    lib.dm_host_pairs(P(vv), P(ff), ctypes.c_int64(nt), P(mm), ctypes.c_int64(n), P(gg), P(lo),
                      P(L), P(F), P(z), P(r), P(cls))
    return F[..., 0] + 1j * F[..., 1], z, r, cls


def _reference(v, f, m, g, box, shape):
    axes = oracle.frequency_axes(box, shape)
    k = (m + (np.array(shape) - 1)) // 2
    xi = np.stack([axes[d][k[:, d]] for d in range(3)], 1)
    xiv = xi @ (v - box[:, 0]).T
    F, dF = oracle.pair_F_and_grads(xiv[:, f[:, 0]], xiv[:, f[:, 1]], xiv[:, f[:, 2]])
    cg = np.conj(g)[:, None]
    z = np.stack([np.real(cg * d) for d in dF], axis=2)
    return F, z, np.real(cg * F)


def _check(hostlib, v, f, m, box, shape, tol_f, tol_z):
    rng = np.random.default_rng(1)
    g = rng.normal(size=len(m)) + 1j * rng.normal(size=len(m))
    F, z, r, cls = _run(hostlib, v, f, m, g, box[:, 0], box[:, 1] - box[:, 0])
    F0, z0, r0 = _reference(v, f, m, g, box, shape)
    assert np.linalg.norm(F - F0) / np.linalg.norm(F0) < tol_f
    assert np.linalg.norm(z - z0) / np.linalg.norm(z0) < tol_z
    assert np.linalg.norm(r - r0) / np.linalg.norm(r0) < tol_f
    for c in (0, 1):  # each path separately
        sel = cls == c
        if sel.sum() > 100:
            assert np.linalg.norm((F - F0)[sel]) / np.linalg.norm(F0[sel]) < tol_f
            assert np.linalg.norm((z - z0)[sel]) / np.linalg.norm(z0[sel]) < tol_z
    return cls


@pytest.mark.parametrize("level,shape", [(2, (21, 21, 21)), (2, (64, 64, 64)),
                                         (4, (128, 128, 128))])
def test_pair_math_matches_oracle(hostlib, level, shape):
    rng = np.random.default_rng(0)
    v, f = icosphere(level, 0.3)
    v, _ = sh_perturb(v, 4, 0.08, rng, radius=0.3)
    box = oracle.compute_box_size(v, 0.2)
    k = np.stack([rng.integers(0, s, 800) for s in shape], 1)
    m = (2 * k - (np.array(shape) - 1)).astype(np.int32)
    sub = rng.choice(len(f), min(len(f), 320), replace=False)
    cls = _check(hostlib, v, f[sub], m, box, shape, 1e-6, 2e-6)
    assert (cls == 0).any() and (cls == 1).any()


def test_pair_math_degenerate_branches(hostlib):
    """Axis-aligned faces on an odd grid: exact zeros in the phase differences."""
    d = load_golden("cube_degenerate")
    box, shape = d["box_size"], tuple(int(s) for s in d["box_shape"])
    k = np.stack(np.unravel_index(d["idx"], shape), 1)
    m = (2 * k - (np.array(shape) - 1)).astype(np.int32)
    cls = _check(hostlib, d["verts"], d["faces"], m, box, shape, 1e-6, 2e-6)
    assert (cls == 2).mean() > 0.01


@pytest.mark.parametrize("scale,shift", [(30.0, (0.0, 0.0, 0.0)), (150.0, (0.9, -0.4, 2.0)),
                                         (600.0, (-3.0, 1.0, 0.5))])
def test_split_phase_off_grid_matches_oracle(hostlib, scale, shift):
    """Off-grid frequencies (explicit xi list): nearest-integer fixed-point phase
    plus the float remainder term, on raw vertex coordinates (lower corner 0,
    length 2.5 max|v|), against the oracle's phases xi . v."""
    rng = np.random.default_rng(3)
    v, f = icosphere(3, 0.3)
    v, _ = sh_perturb(v, 4, 0.08, rng, radius=0.3)
    v = v + np.asarray(shift)
    f = f[rng.choice(len(f), 256, replace=False)]
    xi = rng.normal(size=(500, 3)) * scale
    L = 2.5 * np.abs(v).max(axis=0)
    g = rng.normal(size=len(xi)) + 1j * rng.normal(size=len(xi))
    n, nt = len(xi), len(f)
    F = np.zeros((n, nt, 2), np.float32)
    z = np.zeros((n, nt, 3), np.float32)
    r = np.zeros((n, nt), np.float32)
    cls = np.zeros((n, nt), np.uint8)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    vv, ff = np.ascontiguousarray(v, np.float64), np.ascontiguousarray(f, np.int64)
    xx = np.ascontiguousarray(xi, np.float64)
    gg = np.ascontiguousarray(np.stack([g.real, g.imag], 1), np.float32)
    LL = np.ascontiguousarray(L, np.float64)
    hostlib.dm_host_pairs_off(P(vv), P(ff), ctypes.c_int64(nt), P(xx), ctypes.c_int64(n), P(gg),
                              P(LL), P(F), P(z), P(r), P(cls))
    Fc = F[..., 0] + 1j * F[..., 1]
    xiv = xi @ v.T
    F0, dF = oracle.pair_F_and_grads(xiv[:, f[:, 0]], xiv[:, f[:, 1]], xiv[:, f[:, 2]])
    cg = np.conj(g)[:, None]
    z0 = np.stack([np.real(cg * d) for d in dF], axis=2)
    eF = np.linalg.norm(Fc - F0) / np.linalg.norm(F0)
    ez = np.linalg.norm(z - z0) / np.linalg.norm(z0)
    assert eF < 2e-6 and ez < 4e-6, (eF, ez)


def test_packed_two_pair_series_matches_scalar(hostlib):
    """The paired-FP32 series path (two faces at one frequency in the adjoint, one
    face at two frequencies in the forward) gives the scalar path's results."""
    rng = np.random.default_rng(5)
    v, f = icosphere(4, 0.3)
    v, _ = sh_perturb(v, 4, 0.08, rng, radius=0.3)
    box = oracle.compute_box_size(v, 0.2)
    shape = (96, 96, 96)
    f = f[rng.choice(len(f), 400, replace=False)]
    k = np.stack([rng.integers(20, 76, 300) for _ in range(3)], 1)
    m = (2 * k - (np.array(shape) - 1)).astype(np.int32)
    g = rng.normal(size=len(m)) + 1j * rng.normal(size=len(m))
    F, z, r, cls = _run(hostlib, v, f, m, g, box[:, 0], box[:, 1] - box[:, 0])
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    F2 = np.stack([F.real, F.imag], -1).astype(np.float32).copy()
    z2, r2 = z.copy(), r.copy()
    vv, ff = np.ascontiguousarray(v, np.float64), np.ascontiguousarray(f, np.int64)
    mm = np.ascontiguousarray(m, np.int32)
    gg = np.ascontiguousarray(np.stack([g.real, g.imag], 1), np.float32)
    lo = np.ascontiguousarray(box[:, 0], np.float64)
    L = np.ascontiguousarray(box[:, 1] - box[:, 0], np.float64)
    hostlib.dm_host_series2(P(vv), P(ff), ctypes.c_int64(len(f)), P(mm), ctypes.c_int64(len(m)),
                            P(gg), P(lo), P(L), P(z2), P(r2), P(F2))
    Fp = F2[..., 0] + 1j * F2[..., 1]
    assert (cls == 0).mean() > 0.25
    assert np.linalg.norm(Fp - F) / np.linalg.norm(F) < 1e-6
    assert np.linalg.norm(z2 - z) / np.linalg.norm(z) < 1e-6
    assert np.linalg.norm(r2 - r) / np.linalg.norm(r) < 1e-6
