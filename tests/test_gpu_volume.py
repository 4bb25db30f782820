"""Surface + enclosed-volume ("autofluorescence") transform on the GPU
(deltamic/render.py:228-318) against the reference's golden vectors and the
float64 oracle.  Tolerances (rel-L2, float32 kernels vs float64): ft 1e-5,
vertex gradient 1e-4, regint gradient 1e-5."""
import numpy as np
import pytest
import torch

import oracle.volume as ov
from conftest import band_xi, rel_l2
from deltamic_b200 import (compute_spatial_frequency_grid,
                           fourier_from_mesh_narrowband_autofluorescence, generate_gaussian_psf,
                           ops)
from deltamic_b200.mesh import icosphere, random_sh_shape

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL_FT = 1e-5
TOL_GV = 1e-4
TOL_GR = 1e-5


def _t(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def _axes_otf(shape, lengths, sigma):
    xi = compute_spatial_frequency_grid(shape, lengths, device=DEV, dtype=torch.float32)
    return xi, generate_gaussian_psf(_t(sigma), *xi)


def _band_of(ft_dense, idx):
    return ft_dense.reshape(-1)[torch.as_tensor(idx, device=DEV)].cpu().numpy()


def test_matches_reference_golden(golden_volume):
    name, g = golden_volume
    shape, L = tuple(int(s) for s in g["box_shape"]), g["lengths"]
    xi, otf = _axes_otf(shape, L, g["sigma"])
    V = _t(g["verts"]).requires_grad_(True)
    F = _t(g["faces"], torch.int64)
    R = torch.tensor(float(g["regint"]), device=DEV, requires_grad=True)
    out = fourier_from_mesh_narrowband_autofluorescence(otf, float(g["thresh"]), R, *xi, V, F)
    band = (otf > float(g["thresh"])).reshape(-1).nonzero().reshape(-1).cpu().numpy()
    assert np.array_equal(band, g["idx"])  # same narrow band, index for index
    ft = _band_of(out.detach(), g["idx"])
    ref = g["ft"]
    live = ~np.isnan(ref)
    e = rel_l2(ft[live], ref[live])
    print(f"{name}: ft rel {e:.2e}")
    assert e < TOL_FT
    if not live.all():  # odd grid: the limit 1 - regint where the reference has 0/0
        assert abs(ft[~live][0] - (1.0 - float(g["regint"]))) < 1e-5
    if "w" in g:
        w = torch.zeros(shape, dtype=torch.complex64, device=DEV).reshape(-1)
        w[torch.as_tensor(g["idx"], device=DEV)] = _t(g["w"], torch.complex64)
        loss = torch.sum(torch.real(torch.conj(w.reshape(shape)) * out))
        loss.backward()
        ev = rel_l2(V.grad.cpu().numpy(), g["grad_verts"])
        er = abs(float(R.grad) - float(g["grad_regint"])) / abs(float(g["grad_regint"]))
        print(f"  grad verts rel {ev:.2e}, grad regint rel {er:.2e}")
        assert ev < TOL_GV
        assert er < TOL_GR


@pytest.mark.parametrize("level,shape,herm", [(2, (24, 20, 18), True), (3, (33, 33, 33), True),
                                              (2, (20, 20, 20), False)])
def test_forward_and_adjoint_match_oracle(level, shape, herm):
    """Mirror-symmetric bands (half evaluated) and a lopsided band (all evaluated),
    odd grids with xi = 0 included; a random cotangent on the band."""
    v, f = random_sh_shape(level, 0.3, 4, 0.08, seed=level)
    v = v + np.array([0.05, -0.11, 0.02])
    L = np.array([1.1, 1.0, 0.95])
    xi, otf = _axes_otf(shape, L, np.diag([1e-3, 1.5e-3, 4e-3]))
    if not herm:  # drop one octant's half: the band is no longer closed under xi -> -xi
        otf = otf.clone()
        otf[: shape[0] // 2, : shape[1] // 2, :] *= 0.0
    grid = ops.FreqGrid(np.stack([np.zeros(3), L], axis=1), shape)
    band = ops.narrowband(otf.contiguous(), 1e-5)
    assert ops.band_is_hermitian(band) == herm
    V, F = _t(v), _t(f, torch.int64)
    regint = 0.9
    R = _t([regint])
    ft, vol = ops.volume_list(V, F, R, grid, band)
    idx = band.cpu().numpy().astype(np.int64)
    xil = band_xi(shape, L, idx)
    ft64, vol64 = ov.volume_forward(v, f, regint, xil)
    assert rel_l2(ft.cpu().numpy(), ft64) < TOL_FT
    assert rel_l2(vol.cpu().numpy(), vol64) < TOL_FT
    rng = np.random.default_rng(level)
    g = (rng.normal(size=len(idx)) + 1j * rng.normal(size=len(idx))).astype(np.complex64)
    gv, gr = ops.volume_backward_list(V, F, R, grid, band, ft, vol,
                                      grad_list=_t(g, torch.complex64))
    rv, rr = ov.volume_backward(v, f, regint, xil, g)
    ev, er = rel_l2(gv.cpu().numpy(), rv), abs(float(gr) - rr) / abs(rr)
    print(f"level {level} {shape} herm={herm}: band {len(idx)}, grad verts rel {ev:.2e}, "
          f"regint rel {er:.2e}")
    assert ev < TOL_GV
    assert er < TOL_GR


def test_translation_multiplies_by_a_phase():
    """A closed mesh moved by t: ft(xi) -> exp(-i xi.t) ft(xi) (areas, normals
    and regvol are translation invariant)."""
    v, f = icosphere(3, 0.25)
    shape, L = (24, 24, 24), np.array([1.0, 1.0, 1.0])
    xi, otf = _axes_otf(shape, L, 2e-3 * np.eye(3))
    t = np.array([0.13, -0.07, 0.21])
    F = _t(f, torch.int64)
    a = fourier_from_mesh_narrowband_autofluorescence(otf, 1e-5, 0.7, *xi, _t(v), F)
    b = fourier_from_mesh_narrowband_autofluorescence(otf, 1e-5, 0.7, *xi, _t(v + t), F)
    g0, g1, g2 = torch.meshgrid(*xi, indexing="ij")
    ph = torch.exp(-1j * (g0 * t[0] + g1 * t[1] + g2 * t[2]).double()).to(torch.complex64)
    assert rel_l2((a * ph).cpu().numpy(), b.cpu().numpy()) < 2e-5


def test_empty_band_no_faces_and_float64_inputs():
    v, f = icosphere(1, 0.3)
    shape, L = (16, 16, 16), np.array([1.0, 1.0, 1.0])
    xi, otf = _axes_otf(shape, L, 1e-3 * np.eye(3))
    out = fourier_from_mesh_narrowband_autofluorescence(otf, 2.0, 0.5, *xi, _t(v),
                                                        _t(f, torch.int64))
    assert out.shape == shape and float(out.abs().max()) == 0.0
    none = fourier_from_mesh_narrowband_autofluorescence(
        otf, 1e-5, 0.5, *xi, _t(v), torch.zeros(0, 3, dtype=torch.int64, device=DEV))
    assert float(none.abs().max()) == 0.0
    # float32 only: float64 vertices are refused, not computed in float32
    V64 = torch.tensor(v, dtype=torch.float64, device=DEV, requires_grad=True)
    with pytest.raises(TypeError):
        fourier_from_mesh_narrowband_autofluorescence(otf, 1e-5, 0.5, *xi, V64,
                                                      _t(f, torch.int64))

