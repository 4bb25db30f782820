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


def gibson_lanni_radial(shape, NA=1.4, wavelength=0.610, res_lateral=0.1, res_axial=0.1,
                        ns=1.33, ng0=1.499, ng=1.5, ni0=1.499, ni=1.5, ti0=150, tg0=170,
                        tg=169.99, pZ=2.0, min_wavelength=0.436, num_basis=100):
    """The pupil-phase fit is restated with torch CPU tensors of the reference's
    dtypes: the pupil radius is a float32 linspace and the parameters 0-d float64
    tensors, so by torch's promotion rules OPDs, OPDg, ``ti0 * sqrt(...)`` and the
    axial positions are float32 quantities (psf.py:86, 106-118) -- part of the
    reference's result at the 1e-4 level."""
    nx, ny, nz = shape
    t = lambda v: torch.tensor(v, dtype=torch.double)
    NA_, wl_, ra_ = t(NA), t(wavelength), t(res_axial)
    sf = (NA_ * (3 * torch.arange(1, num_basis + 1, dtype=torch.double) - 2)
          * min_wavelength / wl_)
    rhomax_t = min([NA_, t(ns), t(ni), t(ni0), t(ng), t(ng0)]) / NA_
    rho = torch.linspace(0, rhomax_t.item(), 1000)
    seps = np.sqrt(2.22045e-16)
    sq = lambda n_: torch.sqrt((t(n_) * t(n_) - NA_ * NA_ * rho * rho).clamp(seps))
    zv = (ra_ * torch.arange(-nz / 2, nz / 2) + ra_ / 2).type(torch.double)
    W = 2 * np.pi / wl_ * (t(pZ) * sq(ns) + ((zv.reshape(-1, 1) + t(ti0)) * sq(ni)
                                             - t(ti0) * sq(ni0))
                           + (t(tg) * sq(ng) - t(tg0) * sq(ng0)))
    phase = (torch.cos(W) + 1j * torch.sin(W)).numpy()
    # torch's Bessel functions, as the reference: they differ from scipy's by up to
    # 4e-7, and the least-squares fit below is ill-conditioned (cond(J) ~ 4e12)
    tj0 = lambda x: torch.special.bessel_j0(torch.as_tensor(x)).numpy()
    tj1 = lambda x: torch.special.bessel_j1(torch.as_tensor(x)).numpy()
    J = torch.special.bessel_j0(sf.reshape(-1, 1) * rho).numpy().astype(np.complex128)
    C = np.linalg.lstsq(J.T, phase.T, rcond=None)[0]                 # [K, nz]
    sf, rhomax = sf.numpy(), float(rhomax_t)
    dx = np.arange(nx) - (nx - 1) / 2
    dy = np.arange(ny) - (ny - 1) / 2
    r2 = (dx[:, None] ** 2 + dy[None, :] ** 2).reshape(-1)
    u2, inv = np.unique(r2, return_inverse=True)
    b = 2 * np.pi * np.sqrt(u2) * res_lateral * NA / wavelength
    R = ((sf * tj1(sf * rhomax) * tj0(b[:, None] * rhomax) * rhomax
          - b[:, None] * tj0(sf * rhomax) * tj1(b[:, None] * rhomax) * rhomax)
         / (sf * sf - b[:, None] ** 2))
    prof = np.abs(R @ C) ** 2                                         # [U, nz]
    return (prof[inv] / prof.max()).reshape(nx, ny, nz)


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
