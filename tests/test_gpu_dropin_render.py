"""The reference-named image stage on the device kernels: ``normalize_tensor``
(render.py:5-6) against the eager expression it replaces, and
``render_image_from_ftmesh`` (render.py:177-180) of a ``Fourier3dMesh`` spectrum
(band-box DFTs) against ``abs(ifftn(ftmesh * OTF))`` on cuFFT and a float64
evaluation.  Tolerances: normalize bit-exact at c = 0 (same operation order),
2 ulp otherwise, gradients 1e-6 rel-L2 against the float64 expression; render
image 1e-5 rel-L2 against float64, gradients 1e-4 against the cuFFT route."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from deltamic_b200 import render
from deltamic_b200.mesh import random_sh_shape
from deltamic_b200.psf import generate_gaussian_psf
from deltamic_b200.render import (Fourier3dMesh, compute_box_size, normalize_tensor,
                                  render_image_from_ftmesh)

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _eager(t, c=0):
    lo, hi = t.min(), t.max()
    return ((t - lo) / (hi - lo) + c) / (1 + c)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("c", [0, 0.3])
@pytest.mark.parametrize("shape", [(1,), (7, 5, 3), (96, 80, 72)])
def test_normalize_matches_eager(dtype, c, shape):
    g = torch.Generator(device=DEV).manual_seed(11)
    t = torch.rand(shape, generator=g, device=DEV, dtype=dtype) * 3 - 1
    if t.numel() == 1:  # (t - t) / (t - t): NaN, as the eager expression gives
        assert torch.isnan(normalize_tensor(t, c)).all() and torch.isnan(_eager(t, c)).all()
        return
    t.view(-1)[::17] = t.min()  # ties at the min and the max
    t.view(-1)[5::23] = t.max()
    a = t.clone().requires_grad_(True)
    out = normalize_tensor(a, c)
    ref = _eager(t, c)
    if c == 0:
        assert torch.equal(out, ref)
    else:
        assert torch.max(torch.abs(out - ref)).item() <= 2 * torch.finfo(dtype).eps
    # gradient against the eager expression in float64 (the kernels sum in float64)
    b = t.double().requires_grad_(True)
    w = torch.randn(shape, generator=g, device=DEV, dtype=dtype)
    (out * w).sum().backward()
    (_eager(b, c) * w.double()).sum().backward()
    tol = 1e-6 if dtype == torch.float32 else 1e-12
    assert rel_l2(a.grad.cpu().numpy(), b.grad.cpu().numpy()) < tol
    # the tied elements carry the min / max terms, shared evenly
    for m in (t == t.min(), t == t.max()):
        assert int(m.sum()) > 1
        assert rel_l2(a.grad[m].cpu().numpy(), b.grad[m].cpu().numpy()) < 10 * tol


def test_normalize_nan_and_fallbacks():
    t = torch.linspace(0, 1, 1000, device=DEV)
    t[500] = float("nan")
    assert torch.isnan(normalize_tensor(t)).all() and torch.isnan(_eager(t)).all()
    # a learnable contrast keeps the eager expression and its gradient
    c = torch.tensor(0.2, device=DEV, requires_grad=True)
    x = torch.rand(64, device=DEV)
    normalize_tensor(x, c).sum().backward()
    assert c.grad is not None and torch.isfinite(c.grad)
    # host tensors: the eager expression
    xc = torch.rand(10)
    assert torch.equal(normalize_tensor(xc), _eager(xc))


def _scene(shape, level=3, seed=5, sigma=(1e-3, 1e-3, 4e-3), thresh=1e-5):
    v, f = random_sh_shape(level, 0.3, 4, 0.08, seed=seed)
    c = np.random.default_rng(seed).uniform(0.5, 1.5, len(f))
    box = compute_box_size(v, 0.2)
    fm = Fourier3dMesh(box, shape, device=DEV, dtype=torch.float32, narrowband_thresh=thresh)
    s = torch.tensor(np.diag(sigma), dtype=torch.float32, device=DEV)
    otf = generate_gaussian_psf(s, fm.xi0, fm.xi1, fm.xi2)
    fm.OTF = otf
    return fm, otf, v, f, c


def _dense_image64(ft, otf, shape):
    return torch.abs(torch.fft.ifftn(ft.detach().to(torch.complex128) * otf.double(),
                                     list(shape)))


@pytest.mark.parametrize("shape", [(64, 64, 64), (80, 72, 60), (200, 200, 200)])
def test_render_bandbox_route_matches_dense(shape):
    fm, otf, v, f, c = _scene(shape, level=3 if shape[0] < 200 else 5)
    V = torch.tensor(v, dtype=torch.float32, device=DEV, requires_grad=True)
    F = torch.tensor(f, device=DEV)
    C = torch.tensor(c, dtype=torch.float32, device=DEV, requires_grad=True)
    ft = fm(V, F, C)
    assert render._band_route(ft, otf, shape) is not None  # the band-box DFTs serve it
    img = render_image_from_ftmesh(ft, otf, shape)
    ref = _dense_image64(ft, otf, shape)
    assert img.dtype == torch.float32 and img.shape == tuple(shape)
    assert rel_l2(img.detach().cpu().numpy(), ref.cpu().numpy()) < 1e-5
    # gradients against the same chain on cuFFT (the dense route)
    g = torch.Generator(device=DEV).manual_seed(3)
    w = torch.rand(shape, generator=g, device=DEV)
    (img * w).sum().backward()
    V2 = V.detach().clone().requires_grad_(True)
    C2 = C.detach().clone().requires_grad_(True)
    ft2 = fm(V2, F, C2)
    img2 = torch.abs(torch.fft.ifftn(ft2 * otf, list(shape)))
    (img2 * w).sum().backward()
    assert rel_l2(V.grad.cpu().numpy(), V2.grad.cpu().numpy()) < 1e-4
    assert rel_l2(C.grad.cpu().numpy(), C2.grad.cpu().numpy()) < 1e-4


def test_render_bandbox_otf_gradient_and_fit_loss():
    """A learnable PSF (OTF from log-sigma): vertex, coefficient and log-sigma
    gradients of the band-box route against the cuFFT route for a weighted image
    sum; then the reference's fitting loss, mse(normalize(render), target): same
    value on both routes.  (Its gradient also goes through z/|z| at the image
    minimum, where |z| is near zero and z's direction is float32 rounding noise
    on any route, so the two routes' gradients of that loss are not compared.)"""
    shape = (64, 64, 64)
    fm, _, v, f, c = _scene(shape)
    V = torch.tensor(v * 1.03, dtype=torch.float32, device=DEV)
    F = torch.tensor(f, device=DEV)
    C = torch.tensor(c, dtype=torch.float32, device=DEV)
    with torch.no_grad():
        tgt = normalize_tensor(render_image_from_ftmesh(fm(torch.tensor(
            v, dtype=torch.float32, device=DEV), F, C), fm.OTF, shape))
    w = torch.rand(shape, generator=torch.Generator(device=DEV).manual_seed(9), device=DEV)
    out = {}
    for route in ("bandbox", "dense"):
        Vr = V.clone().requires_grad_(True)
        Cr = C.clone().requires_grad_(True)
        ls = torch.log(torch.tensor([1e-3, 1e-3, 4e-3], device=DEV)).requires_grad_(True)
        otf = generate_gaussian_psf(torch.diag(torch.exp(ls)), fm.xi0, fm.xi1, fm.xi2)
        fm.OTF = otf
        ft = fm(Vr, F, Cr)
        if route == "dense":
            ft = ft * 1  # a new tensor without the band record: the cuFFT route
            assert render._band_route(ft, otf, shape) is None
        else:
            assert render._band_route(ft, otf, shape) is not None
        img = render_image_from_ftmesh(ft, otf, shape)
        (img * w).sum().backward(retain_graph=True)
        loss = ((normalize_tensor(img) - tgt) ** 2).mean()
        out[route] = (float(loss), Vr.grad.cpu().numpy(), Cr.grad.cpu().numpy(),
                      ls.grad.cpu().numpy())
        Vr.grad = None
        loss.backward()
        assert torch.isfinite(Vr.grad).all()
    b, d = out["bandbox"], out["dense"]
    assert abs(b[0] - d[0]) < 1e-5 * abs(d[0])
    assert rel_l2(b[1], d[1]) < 1e-4
    assert rel_l2(b[2], d[2]) < 1e-4
    assert rel_l2(b[3], d[3]) < 1e-4


def test_render_route_falls_back_after_in_place_change():
    shape = (64, 64, 64)
    fm, otf, v, f, c = _scene(shape)
    ft = fm(torch.tensor(v, dtype=torch.float32, device=DEV), torch.tensor(f, device=DEV),
            torch.tensor(c, dtype=torch.float32, device=DEV))
    assert render._band_route(ft, otf, shape) is not None
    ft[0, 0, 0] = 1.0 + 0j  # no longer zero off the band
    assert render._band_route(ft, otf, shape) is None
    img = render_image_from_ftmesh(ft, otf, shape)
    assert rel_l2(img.cpu().numpy(), _dense_image64(ft, otf, shape).cpu().numpy()) < 1e-5
    # a padded box_shape is not the band box's grid either
    assert render._band_route(ft, otf, (70, 64, 64)) is None
    # below 64^3 voxels the dense route is the cheaper one
    fs, os_, vs, f_s, cs = _scene((40, 40, 40))
    fts = fs(torch.tensor(vs, dtype=torch.float32, device=DEV), torch.tensor(f_s, device=DEV),
             torch.tensor(cs, dtype=torch.float32, device=DEV))
    assert render._band_route(fts, os_, (40, 40, 40)) is None
