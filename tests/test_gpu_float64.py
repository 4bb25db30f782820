"""Float64 meshFT (Fourier3dMesh(dtype=float64), the double dispatch of the
reference FFI) against the float64 oracle, both with the reference CPU path's
Seps = sqrt(1.19209e-07) (render.py:64-65).

Tolerances (rel-L2): spectrum 1e-11, vertex and coefficient gradients 1e-8 (the
kernels and the oracle evaluate the same double expressions in different orders;
pairs with phase differences just above Seps amplify rounding by 1/Seps^3 in the
partials).  Against the reference's own CPU float64 chain (golden vectors) the
spectrum agrees to 1e-9."""
import numpy as np
import pytest
import torch

import oracle
from conftest import load_golden, rel_l2
from deltamic_b200 import ops
from deltamic_b200.mesh import random_sh_shape

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL_FT64 = 1e-11
TOL_G64 = 1e-8


def _t(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def _cube():
    d = load_golden("cube_degenerate")
    return d["verts"], d["faces"], d["coeff"], d["box_size"], tuple(int(s) for s in d["box_shape"])


def _sh(level, shape, seed):
    v, f = random_sh_shape(level, 0.3, 4, 0.08, seed)
    c = np.random.default_rng(seed + 1).uniform(0.5, 1.5, len(f))
    return v, f, c, oracle.compute_box_size(v, 0.2), shape


CASES = {"sh_l2": lambda: _sh(2, (24, 20, 18), 3), "sh_l3_odd": lambda: _sh(3, (25, 23, 21), 5),
         "cube": _cube}


@pytest.mark.parametrize("name", sorted(CASES))
def test_float64_grid_band_against_oracle(name):
    v, f, c, box, shape = CASES[name]()
    grid = ops.FreqGrid(box, shape)
    xi = grid.axes(torch.float64, DEV)
    sig = torch.tensor(np.diag([1e-3, 1.5e-3, 3e-3]), dtype=torch.float64, device=DEV)
    g0, g1, g2 = torch.meshgrid(*xi, indexing="ij")
    q = torch.stack([g0, g1, g2], -1)
    otf = torch.exp(-0.5 * torch.einsum("...i,ij,...j->...", q, sig, q)).contiguous()
    band = ops.narrowband(otf, 1e-5)
    V, F, C = _t(v), _t(f, torch.int64), _t(c)
    spec = torch.zeros(shape, dtype=torch.complex128, device=DEV)
    ft = ops.meshft64_list(V, F, C, grid, band, otf=otf, spectrum=spec)
    idx = band.cpu().numpy().astype(np.int64)
    xil = oracle.xi_list_from_band(idx, oracle.frequency_axes(box, shape))
    vs = v - box[:, 0]
    ref = oracle.meshft_forward(vs, f, c, xil, seps=oracle.SEPS_F32)
    assert rel_l2(ft.cpu().numpy(), ref) < TOL_FT64, name
    sp = spec.cpu().numpy().reshape(-1)
    assert rel_l2(sp[idx], ref * otf.cpu().numpy().reshape(-1)[idx]) < TOL_FT64
    mask = np.ones(sp.size, bool)
    mask[idx] = False
    assert np.all(sp[mask] == 0)
    rng = np.random.default_rng(11)
    g = rng.normal(size=len(idx)) + 1j * rng.normal(size=len(idx))
    gv, gc = ops.meshft64_backward_list(V, F, C, ft, grid, band, grad_list=_t(g, torch.complex128))
    rv, rc = oracle.meshft_backward(vs, f, c, xil, g, ref, seps=oracle.SEPS_F32)
    print(name, "float64 vs oracle: ft %.2e verts %.2e coeff %.2e" % (
        rel_l2(ft.cpu().numpy(), ref), rel_l2(gv.cpu().numpy(), rv), rel_l2(gc.cpu().numpy(), rc)))
    assert rel_l2(gv.cpu().numpy(), rv) < TOL_G64, name
    assert rel_l2(gc.cpu().numpy(), rc) < TOL_G64, name


def test_float64_xi_list_off_grid_against_oracle():
    """Explicit frequencies (off any grid, |xi| up to 400) on raw vertex
    coordinates: the forward_fourier3d_cpp convention."""
    v, f, c, box, _ = _sh(3, (8, 8, 8), 9)
    v = v + np.array([1.3, -0.7, 2.1])  # no box shift: phases of the raw coordinates
    rng = np.random.default_rng(3)
    xil = rng.normal(size=(700, 3)) * np.array([60.0, 90.0, 130.0])
    xil[:5] = [[0, 0, 0], [1e-9, 0, 0], [0, 250.0, 0], [400.0, 0, 0], [0, 0, -3e-3]]
    V, F, C = _t(v), _t(f, torch.int64), _t(c)
    X = _t(xil)
    ft = ops.meshft64_list(V, F, C, xi_list=X)
    ref = oracle.meshft_forward(v, f, c, xil, seps=oracle.SEPS_F32)
    assert rel_l2(ft.cpu().numpy(), ref) < TOL_FT64
    g = rng.normal(size=len(xil)) + 1j * rng.normal(size=len(xil))
    gv, gc = ops.meshft64_backward_list(V, F, C, ft, xi_list=X, grad_list=_t(g, torch.complex128))
    rv, rc = oracle.meshft_backward(v, f, c, xil, g, ref, seps=oracle.SEPS_F32)
    assert rel_l2(gv.cpu().numpy(), rv) < TOL_G64
    assert rel_l2(gc.cpu().numpy(), rc) < TOL_G64


@pytest.mark.parametrize("name", ["sphere_l1_sum", "sh_l2_aniso_mse", "cube_degenerate"])
def test_float64_module_chain_against_reference_golden(name):
    """Fourier3dMesh(dtype=float64) -> render_image_from_ftmesh -> normalize ->
    loss -> backward on CUDA, against the reference's float64 CPU chain."""
    import deltamic_b200 as dm
    d = load_golden(name)
    shape = tuple(int(s) for s in d["box_shape"])
    V = _t(d["verts"]).requires_grad_(True)
    C = _t(d["coeff"]).requires_grad_(True)
    S = _t(d["sigma"]).requires_grad_(True)
    mft = dm.Fourier3dMesh(torch.tensor(d["box_size"]), shape, device=DEV, dtype=torch.float64,
                           narrowband_thresh=float(d["thresh"]))
    otf = dm.generate_gaussian_psf(S, mft.xi0, mft.xi1, mft.xi2)
    assert otf.dtype == torch.float64
    mft.OTF = otf.detach()
    ft = mft(V, _t(d["faces"], torch.int64), C)
    assert ft.dtype == torch.complex128
    img = dm.render_image_from_ftmesh(ft, otf, shape)
    nimg = dm.normalize_tensor(img)
    loss = nimg.sum() if str(d["loss_kind"]) == "sum" else torch.mean((nimg - _t(d["target"])) ** 2)
    loss.backward()
    band = mft.band().cpu().numpy()
    assert np.array_equal(band, d["idx"])
    e_ft = rel_l2(ft.detach().reshape(-1).cpu().numpy()[band], d["ft"])
    e_img = rel_l2(img.detach().cpu().numpy(), d["image"])
    ev = rel_l2(V.grad.cpu().numpy(), d["grad_verts"])
    ec = rel_l2(C.grad.cpu().numpy(), d["grad_coeff"])
    es = rel_l2(S.grad.cpu().numpy(), d["grad_sigma"])
    print(name, "float64 module vs reference float64: ft %.2e image %.2e verts %.2e coeff %.2e "
          "sigma %.2e" % (e_ft, e_img, ev, ec, es))
    assert e_ft < 1e-9 and e_img < 1e-9
    assert abs(float(loss.detach()) - float(d["loss"])) < 1e-9 * abs(float(d["loss"]))
    assert ev < 1e-6 and ec < 1e-8 and es < 1e-8


def test_float64_meshftcuda_apply_and_refusals():
    from deltamic_b200.cuda_class import MeshFTCUDA
    from deltamic_b200.render import compute_spatial_frequency_grid
    v, f, c, box, shape = _sh(2, (16, 16, 16), 1)
    vs = v - box[:, 0]
    L = box[:, 1] - box[:, 0]
    xi = compute_spatial_frequency_grid(shape, L, device=DEV, dtype=torch.float64)
    otf = torch.exp(-1e-3 * (xi[0][:, None, None] ** 2 + xi[1][None, :, None] ** 2
                             + xi[2][None, None, :] ** 2) / 2).contiguous()
    V = _t(vs).requires_grad_(True)
    out = MeshFTCUDA.apply(V, _t(f, torch.int64), _t(c), *xi, otf, 1e-5)
    assert out.dtype == torch.complex128
    band = (otf > 1e-5).reshape(-1).cpu().numpy()
    idx = np.nonzero(band)[0]
    xil = oracle.xi_list_from_band(idx, [x.cpu().numpy() for x in xi])
    ref = oracle.meshft_forward(vs, f, c, xil, seps=oracle.SEPS_F32)
    assert rel_l2(out.detach().reshape(-1).cpu().numpy()[idx], ref) < TOL_FT64
    out.abs().sum().backward()
    assert V.grad.dtype == torch.float64 and torch.isfinite(V.grad).all()
    # the autofluorescence transform is float32 only: float64 vertices raise
    from deltamic_b200.render import fourier_from_mesh_narrowband_autofluorescence
    with pytest.raises(TypeError):
        fourier_from_mesh_narrowband_autofluorescence(otf.float(), 1e-5, 0.5,
                                                      *[x.float() for x in xi], _t(vs),
                                                      _t(f, torch.int64))
