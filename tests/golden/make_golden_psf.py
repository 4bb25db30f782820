"""Generate golden vectors for the spatial PSF models by running the reference's
own modules (``deltamic/psf.py``) on the CPU.

Run once in a container that has the reference source checked out (read-only),
with ``$DELTAMIC_REF`` naming its root directory:

    DELTAMIC_REF=<reference checkout> python tests/golden/make_golden_psf.py

Cases: ``Gaussian_psf_logsigma`` (psf.py:590-626), ``Anisotropic_gaussian_psf``
(psf.py:628-665), ``Gibson_Lanni_psf`` (psf.py:23-154, two parameter sets),
``Hanser_psf`` (psf.py:157-371, seeded Zernike coefficients) and the Zernike
polynomials of ``zernike`` / ``noll2degrees`` (psf.py:373-548).  Each stores the
module's inputs, its PSF, a seeded weight volume ``w`` and the gradients of
``sum(w * psf)`` with respect to every parameter torch gives one, as
``psf_<case>.npz`` next to this script.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("DELTAMIC_REF", "")


def _import_reference():
    if not REF or not os.path.isdir(os.path.join(REF, "deltamic")):
        raise SystemExit("set $DELTAMIC_REF to the root of a deltaMic checkout")
    sys.path.insert(0, REF)
    import deltamic.psf as psf  # noqa: E402
    return psf


def _weights(shape, rng, dtype):
    return torch.tensor(rng.normal(size=shape), dtype=dtype)


def _grads(module, names):
    out = {}
    for n in names:
        p = getattr(module, n)
        out["grad_" + n] = (np.zeros(p.shape) if p.grad is None
                            else p.grad.detach().double().numpy())
    return out


def main():
    psf = _import_reference()
    torch.set_num_threads(os.cpu_count() or 1)
    rng = np.random.default_rng(11)
    cases = {}

    shape, size = (20, 18, 16), (1.2, 1.0, 0.8)
    m = psf.Gaussian_psf_logsigma(shape, size, sigma=40.0)
    ls = np.log(np.array([[40.0, 3.0, 1.5], [2.0, 35.0, 2.5], [1.2, 1.8, 60.0]]))
    with torch.no_grad():
        m.logsigma.copy_(torch.tensor(ls, dtype=torch.float32))
    out = m()
    w = _weights(shape, rng, torch.float32)
    (out * w).sum().backward()
    cases["logsigma"] = dict(box_shape=np.array(shape), box_size=np.array(size), logsigma=ls,
                             psf=out.detach().double().numpy(), w=w.double().numpy(),
                             **_grads(m, ["logsigma"]))

    shape, size = (20, 18, 16), (1.0, 1.1, 0.9)
    m = psf.Anisotropic_gaussian_psf(shape, size, sigma=30.0, sigma_z=2.0, eps=0.05)
    with torch.no_grad():
        m.sigma.copy_(torch.tensor([[30.0, 5.0], [3.0, 25.0]]))
    out = m()
    w = _weights(shape, rng, torch.float32)
    (out * w).sum().backward()
    cases["aniso"] = dict(box_shape=np.array(shape), box_size=np.array(size),
                          sigma=np.array([[30.0, 5.0], [3.0, 25.0]]), sigma_z=2.0, eps=0.05,
                          psf=out.detach().double().numpy(), w=w.double().numpy(),
                          **_grads(m, ["sigma", "sigma_z", "eps"]))

    gl_names = ["NA", "wavelength", "res_lateral", "res_axial", "ns", "ng0", "ng", "ni0", "ni",
                "ti0", "tg0", "tg", "pZ"]
    for name, shape, kw in (("gl_default", (32, 32, 16), {}),
                            ("gl_custom", (33, 30, 20),
                             dict(NA=1.3, wavelength=0.52, res_lateral=0.08, res_axial=0.15,
                                  pZ=3.0, tg=170.02))):
        m = psf.Gibson_Lanni_psf(shape, **kw)
        out = m()
        w = _weights(shape, rng, torch.float64)
        (out * w).sum().backward()
        cases[name] = dict(box_shape=np.array(shape), kwargs_keys=np.array(list(kw.keys())),
                           kwargs_vals=np.array([float(v) for v in kw.values()]),
                           psf=out.detach().numpy(), w=w.numpy(), **_grads(m, gl_names))

    shape = (32, 30, 20)
    xi = [torch.zeros(n) for n in shape]
    m = psf.Hanser_psf(shape, *xi, res_axial=0.2)
    pc = rng.normal(size=21) * 0.3
    mc = rng.normal(size=21) * 0.05
    with torch.no_grad():
        m.pcoefs.copy_(torch.tensor(pc, dtype=torch.float32))
        m.mcoefs.copy_(torch.tensor(mc, dtype=torch.float32))
    out = m()
    w = _weights(shape, rng, torch.float32)
    (out * w).sum().backward()
    cases["hanser"] = dict(box_shape=np.array(shape), res_axial=0.2, pcoefs=pc, mcoefs=mc,
                           psf=out.detach().double().numpy(), w=w.double().numpy(),
                           **_grads(m, ["NA", "wavelength", "ni", "res_lateral", "res_axial",
                                        "pcoefs", "mcoefs"]))

    r = np.concatenate([np.linspace(0, 1.2, 61), rng.uniform(0, 1, 200)])
    th = np.concatenate([np.linspace(-np.pi, np.pi, 61), rng.uniform(-np.pi, np.pi, 200)])
    n, mm = psf.noll2degrees(np.arange(1, 67))
    cases["zernike"] = dict(r=r, theta=th, n=n, m=mm,
                            z=psf.zernike(r, th, *psf.noll2degrees(np.arange(1, 67))))

    for name, d in cases.items():
        path = os.path.join(HERE, "psf_" + name + ".npz")
        np.savez_compressed(path, **d)
        print(name, "->", path)


if __name__ == "__main__":
    main()
