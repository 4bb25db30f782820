"""Oracle: spatial PSF models of ``deltamic/psf.py`` in numpy float64.

TEST INFRASTRUCTURE ONLY -- the checker for the CUDA path, never the product.

* ``aniso_gaussian_psf``: ``exp(-u^T S u / (2 D)) / D``, ``D = eps + (|z| s_z)^2``
  (``psf.py:656-661``);
* ``zernike_explicit``: Noll-normalised Zernike polynomials from the explicit sum
  ``R_n^m(r) = sum_s (-1)^s (n-s)! / (s! ((n+m)/2-s)! ((n-m)/2-s)!) r^(n-2s)``
  (the reference evaluates the same polynomial through a Jacobi polynomial,
  ``psf.py:373-392``, 520-548);
* ``gibson_lanni_radial``: the Gibson-Lanni PSF of ``psf.py:77-151`` with the
  Fourier-Bessel amplitude evaluated once per distinct pixel radius and scattered,
  the decomposition the CUDA path uses;
* ``hanser_psf``: the pupil / defocus / obliquity / 2-D inverse FFT /
  ``|fftshift|^2`` chain of ``psf.py:244-365``.

Pinned by golden vectors made by the reference modules themselves
(``tests/golden/make_golden_psf.py``).
"""
from __future__ import annotations

from math import factorial

import numpy as np
import torch


def aniso_gaussian_psf(x, y, z, S, sz, eps):
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    D = eps + (np.abs(Z) * sz) ** 2
    q = X * (S[0, 0] * X + S[0, 1] * Y) + Y * (S[1, 0] * X + S[1, 1] * Y)
    return np.exp(-q / (2 * D)) / D


def zernike_explicit(r, theta, n, m):
    """Z_n^m(r, theta) for scalar degrees (0 outside the unit disk)."""
    r = np.asarray(r, np.float64)
    theta = np.asarray(theta, np.float64)
    am = abs(m)
    if (n - am) % 2:
        return np.zeros_like(r)
    h = (n - am) // 2
    R = np.zeros_like(r)
    for s in range(h + 1):
        R += ((-1) ** s * factorial(n - s)
              / (factorial(s) * factorial((n + am) // 2 - s) * factorial(h - s))) * r ** (n - 2 * s)
    ang = np.sin(am * theta) if m < 0 else np.cos(am * theta)
    norm = np.sqrt(n + 1) if m == 0 else np.sqrt(2 * (n + 1))
    return np.where(r <= 1.0, R * ang * norm, 0.0)


GL_DEFAULTS = dict(NA=1.4, wavelength=0.610, res_lateral=0.1, res_axial=0.1, ns=1.33,
                   ng0=1.499, ng=1.5, ni0=1.499, ni=1.5, ti0=150.0, tg0=170.0, tg=169.99,
                   pZ=2.0)


def gibson_lanni_torch(shape, P, min_wavelength=0.436, num_basis=100):
    """The reference's expressions (psf.py:77-151) as torch ops on the device of the
    0-d float64 tensors ``P`` (keys of ``GL_DEFAULTS``), differentiable by torch's
    autograd as the reference is, with the amplitude formed once per distinct pixel
    radius and scattered.  Its pupil radius is a float32 linspace, so by torch's
    promotion rules OPDs, OPDg, ``ti0 * sqrt(...)`` and the axial positions are
    float32 quantities (psf.py:86, 106-118); its Bessel functions are torch's.  On the
    CPU this is the reference's own computation; on a GPU it is what the reference
    gives there -- torch's CUDA float32 arithmetic and Bessel functions differ from
    its CPU ones in the last digits, which the ill-conditioned fit (cond(J) ~ 4e12)
    carries to 1e-5 of the PSF."""
    nx, ny, nz = shape
    dev = P["NA"].device
    NA, wl = P["NA"], P["wavelength"]
    sf = NA * (3 * torch.arange(1, num_basis + 1, dtype=torch.double, device=dev) - 2) \
        * min_wavelength / wl
    rhomax = min([NA, P["ns"], P["ni"], P["ni0"], P["ng"], P["ng0"]]) / NA
    rho = torch.linspace(0, rhomax.item(), 1000).to(dev)
    seps = np.sqrt(2.22045e-16)
    sq = lambda n_: torch.sqrt((n_ * n_ - NA * NA * rho * rho).clamp(seps))
    zv = (P["res_axial"] * torch.arange(-nz / 2, nz / 2, device=dev)
          + P["res_axial"] / 2).type(torch.double)
    W = 2 * np.pi / wl * (P["pZ"] * sq(P["ns"])
                          + ((zv.reshape(-1, 1) + P["ti0"]) * sq(P["ni"])
                             - P["ti0"] * sq(P["ni0"]))
                          + (P["tg"] * sq(P["ng"]) - P["tg0"] * sq(P["ng0"])))
    phase = torch.cos(W) + 1j * torch.sin(W)
    J = torch.special.bessel_j0(sf.reshape(-1, 1) * rho).type(torch.complex128)
    C = torch.linalg.lstsq(J.T, phase.T).solution                    # [K, nz]
    dx = np.arange(nx) - (nx - 1) / 2
    dy = np.arange(ny) - (ny - 1) / 2
    r2 = (dx[:, None] ** 2 + dy[None, :] ** 2).reshape(-1)
    u2, inv = np.unique(r2, return_inverse=True)
    r_pix = torch.tensor(np.sqrt(u2), dtype=torch.double, device=dev) * P["res_lateral"]
    b = (2 * np.pi * r_pix * NA / wl).reshape(-1, 1)
    j0, j1 = torch.special.bessel_j0, torch.special.bessel_j1
    R = ((sf * j1(sf * rhomax) * j0(b * rhomax) * rhomax
          - b * j0(sf * rhomax) * j1(b * rhomax) * rhomax) / (sf * sf - b * b))
    prof = torch.abs(R.type(torch.complex128) @ C) ** 2                # [U, nz]
    idx = torch.as_tensor(inv.reshape(-1), device=dev)
    return (prof[idx] / torch.max(prof)).reshape(nx, ny, nz)


def gibson_lanni_radial(shape, device="cpu", min_wavelength=0.436, num_basis=100, **kw):
    """Numpy result of :func:`gibson_lanni_torch` for float parameters (defaults of
    the reference module)."""
    P = {k: torch.tensor(float(kw.get(k, v)), dtype=torch.double, device=device)
         for k, v in GL_DEFAULTS.items()}
    return gibson_lanni_torch(shape, P, min_wavelength, num_basis).cpu().numpy()


def _noll(j):
    n = int(np.ceil((-3 + np.sqrt(1 + 8 * j)) / 2))
    jr = j - n * (n + 1) // 2
    m1, m2 = (jr, -(jr - 1)) if n % 4 < 2 else (jr - 1, -jr)
    return n, (m1 if (n - m1) % 2 == 0 else m2)


def hanser_psf(shape, pcoefs, mcoefs, NA=1.4, wavelength=0.610, ni=1.5, res_lateral=0.1,
               res_axial=0.25, condition="sine"):
    nx, ny, nz = shape
    zr = (np.arange(nz) - (nz + 1) // 2) * res_axial
    kx, ky = np.fft.fftfreq(nx), np.fft.fftfreq(ny)
    kxx, kyy = np.meshgrid(kx, ky, indexing="ij")
    phi = np.arctan2(kyy, kxx)
    kr = np.sqrt(kxx ** 2 + kyy ** 2) / res_lateral
    kmag = ni / wavelength
    kz = np.sqrt(np.maximum(kmag ** 2 - kr ** 2, 0.0))
    r = kr * wavelength / NA
    Z = np.array([zernike_explicit(r, phi, *_noll(j + 1)) for j in range(len(pcoefs))])
    phase = np.tensordot(pcoefs, Z, 1)
    mag = np.tensordot(mcoefs, Z, 1)
    pupil = ((kr <= NA / wavelength).astype(np.float64) + mag) * np.exp(1j * phase)
    theta = np.arcsin((kr < kmag) * kr / kmag)
    if condition == "sine":
        pupil = pupil / np.sqrt(np.cos(theta))
    elif condition == "herschel":
        pupil = pupil / np.cos(theta)
    pupils = pupil[None] * np.exp(2j * np.pi * kz[None] * zr[:, None, None])
    field = np.fft.fftshift(np.fft.ifftn(pupils, axes=(1, 2)), axes=(1, 2))
    return np.abs(field.transpose(1, 2, 0)) ** 2
