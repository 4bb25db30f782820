"""The reference FFI names on explicit frequency lists: forward_fourier3d_cpp /
backward_fourier3d_cpp (deltamic/cpp/fourier3d_cuda.cpp:27-65) and MeshFTCUDA on
axes that are not centred grids, against the float64 oracle.

Tolerances (rel-L2, float32 split-phase kernels vs float64): spectrum 1e-5,
vertex gradient 1e-4, coefficient gradient 1e-5 (the grid kernels' tolerances)."""
import numpy as np
import pytest
import torch

import oracle
from conftest import load_golden, rel_l2
from deltamic_b200 import ops
from deltamic_b200.fourier3d_cpp import backward_fourier3d_cpp, forward_fourier3d_cpp
from deltamic_b200.mesh import random_sh_shape

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL_FT, TOL_GV, TOL_GC = 1e-5, 1e-4, 1e-5


def _t(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def _mesh(level=3, seed=2, shift=(0.4, -0.25, 1.3)):
    v, f = random_sh_shape(level, 0.3, 4, 0.08, seed)
    c = np.random.default_rng(seed).uniform(0.5, 1.5, len(f))
    return v + np.asarray(shift), f, c


def _random_xi(n, scale, seed):
    rng = np.random.default_rng(seed)
    xi = rng.normal(size=(n, 3)) * np.asarray(scale)
    xi[:4] = [[0.0, 0.0, 0.0], [1e-5, 0.0, 0.0], [0.0, 0.0, 37.0], [-55.0, 20.0, 3.0]]
    return xi


@pytest.mark.parametrize("scale,level", [((40.0, 40.0, 40.0), 2), ((90.0, 60.0, 150.0), 3),
                                         ((400.0, 400.0, 400.0), 3)])
def test_forward_backward_off_grid_against_oracle(scale, level):
    v, f, c = _mesh(level)
    xi = _random_xi(1500, scale, level)
    V, F, C, X = _t(v), _t(f, torch.int64), _t(c), _t(xi)
    ft = forward_fourier3d_cpp(V, F, C, X)
    assert ft.dtype == torch.complex64 and ft.shape == (len(xi),)
    ref = oracle.meshft_forward(v, f, c, xi)
    e_ft = rel_l2(ft.cpu().numpy(), ref)
    rng = np.random.default_rng(5)
    g = (rng.normal(size=len(xi)) + 1j * rng.normal(size=len(xi))).astype(np.complex64)
    gv = backward_fourier3d_cpp(V, F, C, _t(g, torch.complex64), ft, X)
    rv, rc = oracle.meshft_backward(v, f, c, xi, g, ref)
    gv2, gc = ops.meshft_xi_backward_list(V, F, C, X, _t(g, torch.complex64), ft)
    e_gv, e_gc = rel_l2(gv.cpu().numpy(), rv), rel_l2(gc.cpu().numpy(), rc)
    print(f"off-grid |xi|~{scale}: ft {e_ft:.2e} verts {e_gv:.2e} coeff {e_gc:.2e}")
    # frequencies up to |xi| ~ 700 (m ~ 300 on the cell): the float32 phase
    # differences of large faces lose a little more, the coefficient sums most
    tol_gc = TOL_GC if max(scale) < 300 else 2 * TOL_GC
    assert e_ft < TOL_FT and e_gv < TOL_GV and e_gc < tol_gc
    assert torch.equal(gv, gv2)


def test_xi_list_on_the_grid_matches_grid_kernels():
    """The band's own frequencies through the list path equal the grid path
    (phases shifted by the box corner, undone here)."""
    d = load_golden("sh_l2_aniso_mse")
    v, f, c, box = d["verts"], d["faces"], d["coeff"], d["box_size"]
    shape = tuple(int(s) for s in d["box_shape"])
    grid = ops.FreqGrid(box, shape)
    xi_ax = grid.axes(torch.float32, DEV)
    otf = ops.gaussian_otf(_t(d["sigma"]), *xi_ax)
    band = ops.narrowband(otf, float(d["thresh"]))
    V, F, C = _t(v), _t(f, torch.int64), _t(c)
    ftg = ops.meshft_list(V, F, C, grid, band)
    xil = oracle.xi_list_from_band(band.cpu().numpy().astype(np.int64),
                                   oracle.frequency_axes(box, shape))
    ftx = forward_fourier3d_cpp(_t(v - box[:, 0]), F, C, _t(xil))
    assert rel_l2(ftx.cpu().numpy(), ftg.cpu().numpy()) < 2e-6
    assert rel_l2(ftx.cpu().numpy(), d["ft"]) < TOL_FT


def test_translation_phase_law():
    """Moving every vertex by t multiplies the spectrum by exp(-i xi.t) (the list
    path takes the coordinates as given)."""
    v, f, c = _mesh(3, 4, (0, 0, 0))
    xi = _random_xi(800, (80.0, 80.0, 80.0), 9)
    t = np.array([0.31, -1.7, 2.25])
    a = forward_fourier3d_cpp(_t(v), _t(f, torch.int64), _t(c), _t(xi)).cpu().numpy()
    b = forward_fourier3d_cpp(_t(v + t), _t(f, torch.int64), _t(c), _t(xi)).cpu().numpy()
    assert rel_l2(b, a * np.exp(-1j * (xi @ t))) < 2e-5


def test_cfg1_band_through_the_list_path_against_reference_golden():
    """cfg1 (level-3 icosphere, 64^3): the band's frequency list through
    forward_fourier3d_cpp against the reference's float64 spectrum; the
    reference's own float32 spectrum is printed beside it."""
    d = load_golden("cfg1_icosphere_l3_64")
    box, shape = d["box_size"], tuple(int(s) for s in d["box_shape"])
    xil = oracle.xi_list_from_band(d["idx"].astype(np.int64), oracle.frequency_axes(box, shape))
    ft = forward_fourier3d_cpp(_t(d["verts"] - box[:, 0]), _t(d["faces"], torch.int64),
                               _t(d["coeff"]), _t(xil)).cpu().numpy()
    e = rel_l2(ft, d["ft"])
    print(f"cfg1 list path vs reference float64 {e:.2e}; reference float32 vs float64 "
          f"{rel_l2(d['ft_f32'], d['ft']):.2e}")
    assert e < TOL_FT


def test_meshftcuda_on_non_centred_axes():
    from deltamic_b200.cuda_class import MeshFTCUDA
    v, f, c = _mesh(2, 6, (0.5, 0.5, 0.5))
    axes = [np.linspace(-60.0, 70.0, 14), np.linspace(-50.0, 52.0, 13) ** 1,
            np.sort(np.random.default_rng(1).uniform(-80, 80, 12))]
    xs = [_t(a) for a in axes]
    g0, g1, g2 = np.meshgrid(*axes, indexing="ij")
    filt = np.exp(-(g0 ** 2 + g1 ** 2 + 2 * g2 ** 2) * 3e-4)
    V = _t(v).requires_grad_(True)
    out = MeshFTCUDA.apply(V, _t(f, torch.int64), _t(c), *xs, _t(filt), 1e-2)
    mask = (filt.astype(np.float32) > 1e-2).reshape(-1)
    idx = np.nonzero(mask)[0]
    xil = np.stack([g0.reshape(-1)[idx], g1.reshape(-1)[idx], g2.reshape(-1)[idx]], 1)
    ref = oracle.meshft_forward(v, f, c, xil)
    o = out.detach().reshape(-1).cpu().numpy()
    assert rel_l2(o[idx], ref) < TOL_FT
    assert np.all(o[~mask] == 0)
    rng = np.random.default_rng(2)
    G = (rng.normal(size=filt.shape) + 1j * rng.normal(size=filt.shape)).astype(np.complex64)
    out.backward(_t(G, torch.complex64))
    rv, _ = oracle.meshft_backward(v, f, c, xil, G.reshape(-1)[idx], ref)
    assert rel_l2(V.grad.cpu().numpy(), rv) < TOL_GV


def test_float64_shims_against_oracle():
    v, f, c = _mesh(2, 8)
    xi = _random_xi(600, (70.0, 70.0, 70.0), 3)
    V, F, C, X = (_t(v, torch.float64), _t(f, torch.int64), _t(c, torch.float64),
                  _t(xi, torch.float64))
    ft = forward_fourier3d_cpp(V, F, C, X)
    assert ft.dtype == torch.complex128
    ref = oracle.meshft_forward(v, f, c, xi, seps=oracle.SEPS_F32)
    assert rel_l2(ft.cpu().numpy(), ref) < 1e-11
    g = np.random.default_rng(1).normal(size=len(xi)) + 0.5j
    gv = backward_fourier3d_cpp(V, F, C, _t(g, torch.complex128), ft, X)
    rv, _ = oracle.meshft_backward(v, f, c, xi, g, ref, seps=oracle.SEPS_F32)
    assert rel_l2(gv.cpu().numpy(), rv) < 1e-8


def test_shim_argument_errors():
    v, f, c = _mesh(1, 1)
    V, F, C = _t(v), _t(f, torch.int64), _t(c)
    X = _t(_random_xi(10, (5.0, 5.0, 5.0), 0))
    with pytest.raises(RuntimeError, match="contiguous"):
        forward_fourier3d_cpp(V, F, C, _t(np.zeros((3, 10))).t())
    with pytest.raises(RuntimeError, match="dtype"):
        forward_fourier3d_cpp(V, F, C, X.double())
    ft = forward_fourier3d_cpp(V, F, C, X)
    with pytest.raises(RuntimeError, match="grad_output_list"):
        backward_fourier3d_cpp(V, F, C, ft[:5].contiguous(), ft, X)
    empty = forward_fourier3d_cpp(V, F, C, X[:0].contiguous())
    assert empty.shape == (0,)
