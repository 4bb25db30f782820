"""Spatial PSF models on the GPU against the reference modules' golden vectors
(tests/golden/make_golden_psf.py): the PSF and the gradient of sum(w * psf) with
respect to every parameter the reference differentiates.

Tolerances (rel-L2 / relative): float32 models (Gaussian variants, Hanser) PSF
1e-5, gradients 2e-3 (the reference's own float32 sums over the volume);
Gibson-Lanni (float64): PSF and gradients within 1e-9 of the reference's
expressions with torch autograd on the same device, and the PSF within the
reference's own CPU-to-GPU spread of its CPU result (see the test); the reference's gradients hold the Bessel values constant, and so
does the default module (exact_bessel_grad=True is checked against finite
differences)."""
import numpy as np
import pytest
import torch

import oracle.psf as op
from conftest import load_golden, rel_l2
from deltamic_b200 import (Anisotropic_gaussian_psf, Gaussian_psf_logsigma, Gibson_Lanni_psf,
                           Hanser_psf, noll2degrees, zernike)

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _rel(a, b):
    a, b = float(a), float(b)
    return abs(a - b) / max(abs(b), 1e-12)


def _w(g, dtype):
    return torch.tensor(g["w"], dtype=dtype, device=DEV)


def test_logsigma_matches_reference():
    g = load_golden("psf_logsigma")
    m = Gaussian_psf_logsigma(tuple(g["box_shape"]), g["box_size"], sigma=40.0, device=DEV)
    with torch.no_grad():
        m.logsigma.copy_(torch.tensor(g["logsigma"], dtype=torch.float32))
    out = m()
    assert rel_l2(out.detach().cpu().numpy(), g["psf"]) < 1e-5
    (out * _w(g, torch.float32)).sum().backward()
    e = rel_l2(m.logsigma.grad.cpu().numpy(), g["grad_logsigma"])
    print(f"logsigma grad rel {e:.2e}")
    assert e < 2e-3


def test_aniso_matches_reference():
    g = load_golden("psf_aniso")
    m = Anisotropic_gaussian_psf(tuple(g["box_shape"]), g["box_size"], sigma=30.0, sigma_z=2.0,
                                 eps=0.05, device=DEV)
    with torch.no_grad():
        m.sigma.copy_(torch.tensor(g["sigma"], dtype=torch.float32))
    out = m()
    assert rel_l2(out.detach().cpu().numpy(), g["psf"]) < 1e-5
    (out * _w(g, torch.float32)).sum().backward()
    es = rel_l2(m.sigma.grad.cpu().numpy(), g["grad_sigma"])
    ez, ee = _rel(m.sigma_z.grad, g["grad_sigma_z"]), _rel(m.eps.grad, g["grad_eps"])
    print(f"aniso grads rel: sigma {es:.2e} sigma_z {ez:.2e} eps {ee:.2e}")
    assert max(es, ez, ee) < 2e-3


GL_PARAMS = ["NA", "wavelength", "res_lateral", "res_axial", "ns", "ng0", "ng", "ni0", "ni",
             "ti0", "tg0", "tg", "pZ"]


@pytest.mark.parametrize("case", ["psf_gl_default", "psf_gl_custom"])
def test_gibson_lanni_matches_reference(case):
    """Against the oracle's restatement of the reference's expressions evaluated on
    the same GPU with torch autograd (the reference run there): PSF within 1e-9 and
    every parameter gradient within ten times the gradient's own sensitivity to the
    order of its sums (measured on the CPU; 3e-13 for the custom set, 9e-5 for the
    defaults) or within the reference's own CPU-to-GPU spread of that gradient,
    plus 1e-9.  Against the reference run on the CPU (golden):
    within twice the distance between that restatement on the GPU and on the CPU
    -- the reference's own CPU-to-GPU spread (float32 steps in its pupil phase,
    Bessel functions, least squares with cond(J) ~ 4e12) -- plus 1e-9."""
    g = load_golden(case)
    kw = {str(k): float(v) for k, v in zip(g["kwargs_keys"], g["kwargs_vals"])}
    shape = tuple(int(v) for v in g["box_shape"])
    m = Gibson_Lanni_psf(shape, device=DEV, **kw)
    out = m()
    assert out.dtype == torch.float64
    w = _w(g, torch.float64)
    (out * w).sum().backward()
    P = {k: torch.tensor(kw.get(k, v), dtype=torch.float64, device=DEV, requires_grad=True)
         for k, v in op.GL_DEFAULTS.items()}
    same = op.gibson_lanni_torch(shape, P)
    (same * w).sum().backward()
    got, ref_dev = out.detach().cpu().numpy(), same.detach().cpu().numpy()
    spread = rel_l2(ref_dev, g["psf"])
    e_dev, e = rel_l2(got, ref_dev), rel_l2(got, g["psf"])
    eg_dev = {p: _rel(getattr(m, p).grad, P[p].grad) for p in GL_PARAMS}
    eg_spread = {p: _rel(P[p].grad, g["grad_" + p]) for p in GL_PARAMS}
    # how far the reference's gradient moves on the CPU when only the order of its
    # sums changes (the radial restatement against the reference itself): the
    # ill-conditioned least squares magnifies rounding in its backward
    Pc = {k: torch.tensor(kw.get(k, v), dtype=torch.float64, requires_grad=True)
          for k, v in op.GL_DEFAULTS.items()}
    (op.gibson_lanni_torch(shape, Pc) * w.cpu()).sum().backward()
    floor_g = max(_rel(Pc[p].grad, g["grad_" + p]) for p in GL_PARAMS)
    print(f"{case}: psf rel {e_dev:.2e} to the same-device reference expressions, {e:.2e} to "
          f"the CPU reference (its CPU-GPU spread {spread:.2e}); grads rel to the same-device "
          "expressions " + " ".join(f"{k} {v:.1e}" for k, v in eg_dev.items())
          + "; the reference's own CPU-GPU gradient spread "
          + " ".join(f"{k} {v:.1e}" for k, v in eg_spread.items()))
    print(f"  gradient floor (order of sums, CPU) {floor_g:.1e}")
    assert e_dev < 1e-9
    assert e < 2 * spread + 1e-9
    # each gradient: within the reordering floor, or within the reference's own
    # CPU-to-GPU spread for that parameter (torch's GPU backward sums with atomics)
    for p in GL_PARAMS:
        assert eg_dev[p] < max(10 * floor_g, eg_spread[p]) + 1e-9, p


@pytest.mark.parametrize("param", ["wavelength", "res_lateral"])
def test_gibson_lanni_exact_gradient_matches_finite_differences(param):
    """exact_bessel_grad=True: the full derivative through the fit's and the basis's
    Bessel values, against a central difference of the float64 forward
    (well-conditioned parameters).  Parameters that the reference combines with
    its float32 pupil radius (NA, pZ, the thicknesses and indices) carry float32
    rounding in the forward, which a 1e-6 step cannot resolve."""
    kw = dict(NA=1.3, wavelength=0.52, res_lateral=0.08, res_axial=0.15, pZ=3.0, tg=170.02)
    shape = (21, 20, 8)
    w = torch.tensor(np.random.default_rng(3).normal(size=shape), device=DEV)
    m = Gibson_Lanni_psf(shape, device=DEV, exact_bessel_grad=True, **kw)
    (m() * w).sum().backward()
    g = float(getattr(m, param).grad)
    h = 1e-6 * kw[param]
    f = []
    for sgn in (1, -1):
        mm = Gibson_Lanni_psf(shape, device=DEV, **dict(kw, **{param: kw[param] + sgn * h}))
        with torch.no_grad():
            f.append(float((mm() * w).sum()))
    fd = (f[0] - f[1]) / (2 * h)
    print(f"{param}: autograd {g:.6e} central difference {fd:.6e}")
    assert abs(g - fd) <= 1e-4 * max(abs(fd), 1e-6 * abs(g) + 1e-12)


def test_hanser_matches_reference():
    g = load_golden("psf_hanser")
    shape = tuple(int(v) for v in g["box_shape"])
    xi = [torch.zeros(n, device=DEV) for n in shape]
    m = Hanser_psf(shape, *xi, device=DEV, res_axial=float(g["res_axial"]))
    with torch.no_grad():
        m.pcoefs.copy_(torch.tensor(g["pcoefs"], dtype=torch.float32))
        m.mcoefs.copy_(torch.tensor(g["mcoefs"], dtype=torch.float32))
    out = m()
    e = rel_l2(out.detach().cpu().numpy(), g["psf"])
    (out * _w(g, torch.float32)).sum().backward()
    ec = {p: rel_l2(getattr(m, p).grad.cpu().numpy(), g["grad_" + p])
          for p in ("pcoefs", "mcoefs")}
    es = {p: _rel(getattr(m, p).grad, g["grad_" + p])
          for p in ("wavelength", "ni", "res_lateral", "res_axial")}
    print(f"hanser: psf rel {e:.2e}; grads rel {ec} {es}")
    assert e < 1e-5
    assert max(ec.values()) < 2e-3 and max(es.values()) < 2e-3


def test_zernike_kernel_matches_reference():
    g = load_golden("psf_zernike")
    n, m = noll2degrees(np.arange(1, 67))
    r = torch.tensor(g["r"], dtype=torch.float32, device=DEV)
    th = torch.tensor(g["theta"], dtype=torch.float32, device=DEV)
    Z = zernike(r, th, n, m).cpu().numpy()
    # float32 inputs: compare with the float64 polynomials at the same float32 points
    ref = np.array([op.zernike_explicit(r.cpu().numpy().astype(np.float64),
                                        th.cpu().numpy().astype(np.float64), a, b)
                    for a, b in zip(n, m)])
    assert np.max(np.abs(Z - ref)) < 2e-6 * max(1.0, np.abs(ref).max())
    assert rel_l2(Z, g["z"]) < 1e-5
