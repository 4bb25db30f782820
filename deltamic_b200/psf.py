"""PSF / OTF generators of deltaMic (``deltamic/psf.py``) on the B200 kernels.

* ``generate_gaussian_psf(sigma, xi0, xi1, xi2)`` (psf.py:15-20) returns
  ``exp(-(xi^T S xi)/2)`` on the outer grid of the axes, differentiable in
  ``sigma`` (a [3,3] CUDA tensor); ``generate_gaussian_psf_from_sigma``
  (psf.py:8-12) is the isotropic form ``exp(-s |xi|^2 / 2)``.
* ``Gaussian_psf(box_shape, box_size, sigma, device, with_grad, dtype)``
  (psf.py:551-587): the spatial Gaussian PSF module of the reference notebook, on
  ``linspace(-box_size[d]/2, box_size[d]/2, box_shape[d])`` axes, with a learnable
  [3,3] ``sigma``; the same kernel as the Gaussian OTF evaluates it.
* ``otf_from_psf(psf)``: the notebook's ``torch.abs(torch.fft.fftshift(
  torch.fft.fftn(PSF)))`` (Examples/Gradient_Descent.ipynb cell 2) with its
  gradient to the PSF: cuFFT for the 3-D transform, the library's fused
  shift-and-modulus kernels around it.
* ``Gaussian_psf_logsigma`` (psf.py:590-626) and ``Anisotropic_gaussian_psf``
  (psf.py:628-665);
* ``Gibson_Lanni_psf`` (psf.py:23-154): the pupil-phase fit (OPDs, Bessel basis,
  least squares) runs as torch ops on the parameters; the Fourier-Bessel basis is
  formed for the distinct pixel radii only and the normalised intensity is
  scattered to the volume by the library's kernels (radial symmetry), with the
  products ``R @ C`` on cuBLAS;
* ``Hanser_psf`` (psf.py:157-371) with ``zernike`` / ``noll2degrees``
  (psf.py:373-548): Zernike polynomials, the defocused pupil planes and the
  shifted intensity are library kernels around cuFFT's batched 2-D inverse FFT.

Every module takes its parameters as ``nn.Parameter`` with gradients, like the
reference; they run on CUDA devices only.
"""
from __future__ import annotations

import numpy as np
import torch
from torch import nn

from . import _native as N
from . import ops

__all__ = ["generate_gaussian_psf", "generate_gaussian_psf_from_sigma", "Gaussian_psf",
           "Gaussian_psf_logsigma", "Anisotropic_gaussian_psf", "Gibson_Lanni_psf",
           "Hanser_psf", "zernike", "noll2degrees", "otf_from_psf"]


def generate_gaussian_psf(sigma, xi0, xi1, xi2):
    """exp(-(xi^T sigma xi)/2) on the grid of the axes with gradients to sigma: the
    float64 kernel for a float64 sigma or float64 axes, else the float32 one."""
    return ops.gaussian_otf(sigma, xi0, xi1, xi2)


def generate_gaussian_psf_from_sigma(sigma, xi0, xi1, xi2):
    s = torch.as_tensor(sigma, dtype=torch.float32, device=xi0.device)
    return ops.gaussian_otf(s * torch.eye(3, device=xi0.device), xi0, xi1, xi2)


class Gaussian_psf(nn.Module):
    """Spatial Gaussian PSF exp(-(x^T sigma x)/2) on a centred linspace grid."""

    def __init__(self, box_shape, box_size, sigma=1, device="cuda", with_grad=True,
                 dtype=torch.float):
        super().__init__()
        if torch.device(device).type != "cuda":
            raise RuntimeError("deltamic_b200.Gaussian_psf runs on CUDA devices only")
        self.with_grad = with_grad
        self.dtype = dtype
        self.device = device
        self.axes = _linspace_axes(box_shape, box_size, device, _real(dtype))
        self.sigma = nn.Parameter(torch.tensor(np.identity(3) * sigma, dtype=dtype,
                                               device=device), requires_grad=with_grad)

    def forward(self):
        # float64 parameters run the float64 kernel, anything else the float32 one
        return ops.gaussian_otf(self.sigma.to(_real(self.dtype)), *self.axes)


class _OTFfromPSF(torch.autograd.Function):
    @staticmethod
    def forward(ctx, psf):
        F = torch.fft.fftn(psf.to(torch.complex64))
        n = psf.shape
        otf = torch.empty(n, dtype=torch.float32, device=psf.device)
        N.check(N.lib().dm_otf_from_spectrum(N.ptr(F), n[0], n[1], n[2], N.ptr(otf),
                                             N.stream_ptr(psf.device)), "dm_otf_from_spectrum")
        ctx.save_for_backward(F)
        return otf

    @staticmethod
    def backward(ctx, g):
        (F,) = ctx.saved_tensors
        n = F.shape
        gF = torch.empty_like(F)
        N.check(N.lib().dm_otf_from_spectrum_backward(
            N.ptr(F), N.ptr(g.contiguous().float()), n[0], n[1], n[2], N.ptr(gF),
            N.stream_ptr(F.device)), "dm_otf_from_spectrum_backward")
        # adjoint of the unnormalised forward transform: numel * ifftn, real part
        return (torch.fft.ifftn(gF) * gF.numel()).real


def otf_from_psf(psf: torch.Tensor) -> torch.Tensor:
    """|fftshift(fftn(psf))| (float32, box_shape), differentiable in ``psf``."""
    N.require_cuda(psf, "PSF")
    if psf.dim() != 3:
        raise ValueError("PSF must be a 3-D tensor")
    return _OTFfromPSF.apply(psf.contiguous().float())


def _cuda_only(device, name):
    if torch.device(device).type != "cuda":
        raise RuntimeError(f"deltamic_b200.{name} runs on CUDA devices only")


def _real(dtype):
    return torch.float64 if dtype == torch.float64 else torch.float32


def _linspace_axes(box_shape, box_size, device, dtype=torch.float32):
    L = np.asarray(torch.as_tensor(box_size).detach().cpu().double().numpy(), np.float64)
    return tuple(torch.linspace(-L[d] / 2, L[d] / 2, int(box_shape[d]), dtype=dtype,
                                device=device) for d in range(3))


class Gaussian_psf_logsigma(nn.Module):
    """``exp(-(x^T S x)/2)`` with ``S = exp(logsigma)`` elementwise (psf.py:590-626;
    the off-diagonal entries of the initial ``logsigma`` are 0, so S starts with
    ones there, as in the reference)."""

    def __init__(self, box_shape, box_size, sigma=1, device="cuda", with_grad=True,
                 dtype=torch.float):
        super().__init__()
        _cuda_only(device, "Gaussian_psf_logsigma")
        self.with_grad = with_grad
        self.dtype = dtype
        self.device = device
        self.axes = _linspace_axes(box_shape, box_size, device, _real(dtype))
        self.logsigma = nn.Parameter(torch.tensor(np.identity(3) * np.log(sigma), dtype=dtype,
                                                  device=device), requires_grad=with_grad)

    def forward(self):
        self.sigma = torch.exp(self.logsigma)
        return ops.gaussian_otf(self.sigma.to(_real(self.dtype)), *self.axes)


class _AnisoPSF(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, x, y, z):
        n = (x.numel(), y.numel(), z.numel())
        psf = torch.empty(n, dtype=torch.float32, device=params.device)
        N.check(N.lib().dm_aniso_gaussian_psf(N.ptr(params), N.ptr(x), n[0], N.ptr(y), n[1],
                                              N.ptr(z), n[2], N.ptr(psf),
                                              N.stream_ptr(params.device)),
                "dm_aniso_gaussian_psf")
        ctx.save_for_backward(params, x, y, z, psf)
        return psf

    @staticmethod
    def backward(ctx, g):
        params, x, y, z, psf = ctx.saved_tensors
        lib = N.lib()
        gp = torch.empty(6, dtype=torch.float32, device=params.device)
        ws = N.WORKSPACES.get("aniso", lib.dm_aniso_gaussian_psf_grad_workspace_size(psf.numel()),
                              params.device)
        N.check(lib.dm_aniso_gaussian_psf_grad(
            N.ptr(g.contiguous().float()), N.ptr(psf), N.ptr(params), N.ptr(x), x.numel(),
            N.ptr(y), y.numel(), N.ptr(z), z.numel(), N.ptr(gp), N.ptr(ws), ws.numel(),
            N.stream_ptr(params.device)), "dm_aniso_gaussian_psf_grad")
        return gp, None, None, None


class Anisotropic_gaussian_psf(nn.Module):
    """``exp(-u^T S u / (2 D)) / D``, ``u = (x, y)``, ``D = eps + (|z| sigma_z)^2``
    (psf.py:628-665) with learnable [2,2] ``sigma``, ``sigma_z`` and ``eps``."""

    def __init__(self, box_shape, box_size, sigma=1, sigma_z=1, eps=0.01, device="cuda",
                 with_grad=True, dtype=torch.float):
        super().__init__()
        _cuda_only(device, "Anisotropic_gaussian_psf")
        self.with_grad = with_grad
        self.dtype = dtype
        self.device = device
        self.axes = _linspace_axes(box_shape, box_size, device)
        mk = lambda v: nn.Parameter(torch.tensor(v, dtype=dtype, device=device),
                                    requires_grad=with_grad)
        self.sigma = mk(np.identity(2) * sigma)
        self.sigma_z = mk(sigma_z)
        self.eps = mk(eps)

    def forward(self):
        params = torch.cat([self.sigma.reshape(4), self.sigma_z.reshape(1),
                            self.eps.reshape(1)]).float().contiguous()
        out = _AnisoPSF.apply(params, *self.axes)
        return out.to(self.dtype) if self.dtype != torch.float32 else out


# ---------------------------------------------------------------------------
# Gibson-Lanni

_RADIAL: dict = {}


def _radial_tables(nx, ny, device):
    """Distinct pixel distances from the lateral centre ((n-1)/2, psf.py:79-80),
    the radius index of every pixel, and the pixels of every radius (CSR)."""
    key = (nx, ny, str(device))
    hit = _RADIAL.get(key)
    if hit is not None:
        return hit
    dx = np.arange(nx, dtype=np.float64) - (nx - 1) / 2
    dy = np.arange(ny, dtype=np.float64) - (ny - 1) / 2
    r2 = (dx[:, None] ** 2 + dy[None, :] ** 2).reshape(-1)
    u2, inv = np.unique(r2, return_inverse=True)
    order = np.argsort(inv, kind="stable")
    off = np.zeros(len(u2) + 1, np.int64)
    np.add.at(off, inv + 1, 1)
    off = np.cumsum(off)
    t = (torch.tensor(np.sqrt(u2), dtype=torch.float64, device=device),
         torch.tensor(inv.astype(np.int32), device=device),
         torch.tensor(off.astype(np.int32), device=device),
         torch.tensor(order.astype(np.int32), device=device))
    _RADIAL[key] = t
    return t


class _BesselJ0(torch.autograd.Function):
    """J0 of the pupil fit with its derivative -J1 (torch's bessel_j0 has none)."""

    @staticmethod
    def forward(ctx, x):
        ctx.save_for_backward(x)
        return torch.special.bessel_j0(x)

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        return -torch.special.bessel_j1(x) * g


class _RadialBasis(torch.autograd.Function):
    @staticmethod
    def forward(ctx, scaling, rhomax, b, bess_s, bess_b, exact):
        lib = N.lib()
        K, U = scaling.numel(), b.numel()
        R = torch.empty(U, K, dtype=torch.float64, device=scaling.device)
        N.check(lib.dm_radial_basis(N.ptr(scaling), K, N.ptr(rhomax), N.ptr(b), U, N.ptr(bess_s),
                                    N.ptr(bess_b), N.ptr(R), N.stream_ptr(scaling.device)),
                "dm_radial_basis")
        ctx.save_for_backward(scaling, rhomax, b, bess_s, bess_b)
        ctx.exact = int(bool(exact))
        return R

    @staticmethod
    def backward(ctx, gR):
        scaling, rhomax, b, bess_s, bess_b = ctx.saved_tensors
        lib = N.lib()
        K, U = scaling.numel(), b.numel()
        gs, gr, gb = torch.empty_like(scaling), torch.empty_like(rhomax), torch.empty_like(b)
        ws = N.WORKSPACES.get("rbasis", lib.dm_radial_basis_grad_workspace_size(U, K),
                              scaling.device)
        N.check(lib.dm_radial_basis_grad(N.ptr(gR.contiguous()), N.ptr(scaling), K, N.ptr(rhomax),
                                         N.ptr(b), U, N.ptr(bess_s), N.ptr(bess_b), ctx.exact,
                                         N.ptr(gs), N.ptr(gr), N.ptr(gb), N.ptr(ws), ws.numel(),
                                         N.stream_ptr(scaling.device)), "dm_radial_basis_grad")
        return gs, gr, gb, None, None, None


class _RadialIntensity(torch.autograd.Function):
    @staticmethod
    def forward(ctx, amp, pix, off, pixels, nx, ny):
        lib = N.lib()
        U, nz = amp.shape
        psf = torch.empty(nx, ny, nz, dtype=torch.float64, device=amp.device)
        prof = torch.empty(U, nz, dtype=torch.float64, device=amp.device)
        peak = torch.empty(1, dtype=torch.float64, device=amp.device)
        ws = N.WORKSPACES.get("rint", lib.dm_radial_intensity_workspace_size(U, nz), amp.device)
        N.check(lib.dm_radial_intensity(N.ptr(amp), U, nz, N.ptr(pix), nx * ny, N.ptr(psf),
                                        N.ptr(prof), N.ptr(peak), N.ptr(ws), ws.numel(),
                                        N.stream_ptr(amp.device)), "dm_radial_intensity")
        ctx.save_for_backward(amp, prof, peak, off, pixels)
        return psf

    @staticmethod
    def backward(ctx, g):
        amp, prof, peak, off, pixels = ctx.saved_tensors
        lib = N.lib()
        U, nz = amp.shape
        ga = torch.empty_like(amp)
        ws = N.WORKSPACES.get("rint", lib.dm_radial_intensity_workspace_size(U, nz), amp.device)
        N.check(lib.dm_radial_intensity_backward(
            N.ptr(g.contiguous().double()), N.ptr(amp), N.ptr(prof), N.ptr(peak), U, nz,
            N.ptr(off), N.ptr(pixels), N.ptr(ga), N.ptr(ws), ws.numel(),
            N.stream_ptr(amp.device)), "dm_radial_intensity_backward")
        return ga, None, None, None, None, None


class Gibson_Lanni_psf(nn.Module):
    """Gibson-Lanni PSF by a Fourier-Bessel fit of the pupil phase (psf.py:23-154;
    the method of kmdouglass.github.io's fast Gibson-Lanni solver), float64, with
    gradients to every optical parameter.  ``num_samples`` is 1000 whatever is
    passed, as in the reference (psf.py:75); ``M`` is accepted and unused.

    The reference's gradients treat every Bessel value as a constant (torch's
    ``bessel_j0`` / ``bessel_j1`` have no derivative), so its NA, wavelength and
    res_lateral gradients are partial derivatives; this module returns the same by
    default and the full derivative with ``exact_bessel_grad=True``."""

    def __init__(self, box_shape, NA=1.4, M=100., wavelength=0.610, res_lateral=0.1,
                 res_axial=0.1, ns=1.33, ng0=1.499, ng=1.5, ni0=1.499, ni=1.5, ti0=150,
                 tg0=170, tg=169.99, pZ=2.0, min_wavelength=0.436, num_basis=100,
                 num_samples=1000, device="cuda", exact_bessel_grad=False):
        super().__init__()
        _cuda_only(device, "Gibson_Lanni_psf")
        self.exact_bessel_grad = exact_bessel_grad
        self.device = device
        mk = self.make_param
        self.NA, self.wavelength = mk(NA), mk(wavelength)
        self.res_lateral, self.res_axial = mk(res_lateral), mk(res_axial)
        self.ns, self.ng0, self.ng, self.ni0, self.ni = mk(ns), mk(ng0), mk(ng), mk(ni0), mk(ni)
        self.ti0, self.tg0, self.tg, self.pZ = mk(ti0), mk(tg0), mk(tg), mk(pZ)
        self.size_x, self.size_y, self.size_z = (int(s) for s in box_shape)
        self.eps = 2.22045e-16
        self.Seps = np.sqrt(self.eps)
        self.min_wavelength = min_wavelength
        self.num_basis = num_basis
        self.num_samples = 1000

    def make_param(self, x):
        return nn.Parameter(torch.tensor(x, dtype=torch.double, device=self.device,
                                         requires_grad=True))

    def forward(self):
        dev = self.device
        NA, lam = self.NA, self.wavelength
        scaling = NA * (3 * torch.arange(1, self.num_basis + 1, device=dev, dtype=torch.double)
                        - 2) * self.min_wavelength / lam
        rhomax = min([NA, self.ns, self.ni, self.ni0, self.ng, self.ng0]) / NA
        # the reference's float32 sample points (torch's CPU linspace), moved over
        rho = torch.linspace(0, rhomax.item(), self.num_samples).to(dev)
        with torch.no_grad():  # the reference's five domain asserts, read back once
            lows = torch.stack([(n_ * n_ - NA * NA * r_ * r_).min() for n_, r_ in (
                (self.ns, rhomax), (self.ni, rhomax), (self.ni0, rho), (self.ns, rho),
                (self.ng0, rho))])
            assert float(lows.min()) >= -self.Seps
        zv = (self.res_axial * torch.arange(-self.size_z / 2, self.size_z / 2, device=dev)
              + self.res_axial / 2).type(torch.double)
        na2r2 = NA * NA * rho * rho
        sq = lambda n_: torch.sqrt((n_ * n_ - na2r2).clamp(self.Seps))
        OPDs = self.pZ * sq(self.ns)
        OPDi = (zv.reshape(-1, 1) + self.ti0) * sq(self.ni) - self.ti0 * sq(self.ni0)
        OPDg = self.tg * sq(self.ng) - self.tg0 * sq(self.ng0)
        W = 2 * np.pi / lam * (OPDs + OPDi + OPDg)
        phase = torch.cos(W) + 1j * torch.sin(W)
        x = scaling.reshape(-1, 1) * rho
        J = (_BesselJ0.apply(x) if self.exact_bessel_grad
             else torch.special.bessel_j0(x)).type(torch.complex128)
        C = torch.linalg.lstsq(J.T, phase.T).solution                  # [K, nz]
        radii, pix, off, pixels = _radial_tables(self.size_x, self.size_y, dev)
        b = 2 * np.pi * (radii * self.res_lateral) * NA / lam          # per distinct radius
        with torch.no_grad():  # the Bessel values the fit and the basis share
            sr, br = scaling * rhomax, b * rhomax
            bess_s = torch.cat([torch.special.bessel_j0(sr), torch.special.bessel_j1(sr)])
            bess_b = torch.cat([torch.special.bessel_j0(br), torch.special.bessel_j1(br)])
        R = _RadialBasis.apply(scaling.contiguous(), rhomax.reshape(1).contiguous(),
                               b.contiguous(), bess_s, bess_b, self.exact_bessel_grad)
        amp = (R.type(torch.complex128) @ C).contiguous()             # cuBLAS
        return _RadialIntensity.apply(amp, pix, off, pixels, self.size_x, self.size_y)


# ---------------------------------------------------------------------------
# Zernike polynomials and the Hanser PSF

def noll2degrees(j):
    """Noll index -> (n, m) (psf.py:407-453), vectorised like the reference."""
    j = np.asarray(j)
    if not (j > 0).all():
        raise ValueError("Invalid Noll index")
    n = np.ceil((-3 + np.sqrt(1 + 8 * j)) / 2).astype(int)
    jr = j - (n * (n + 1) / 2).astype(int)
    low = (n % 4) < 2
    m1 = np.where(low, jr, jr - 1)
    m2 = np.where(low, -(jr - 1), -jr)
    m = np.where((n - m1) % 2 == 0, m1, m2)
    return n, m


def _zernike_gpu(r: torch.Tensor, theta: torch.Tensor, n, m) -> torch.Tensor:
    n = np.atleast_1d(np.asarray(n)).ravel()
    m = np.atleast_1d(np.asarray(m)).ravel()
    if n.shape != m.shape:
        raise ValueError("Radial and Azimuthal degrees have different shapes")
    if not (n >= np.abs(m)).all():
        raise ValueError("n must always be greater or equal to m")
    r = r.detach().float().contiguous()
    theta = theta.detach().float().contiguous()
    deg = np.ascontiguousarray(np.stack([n, m], axis=1).astype(np.int32).ravel())
    out = torch.empty((len(n),) + tuple(r.shape), dtype=torch.float32, device=r.device)
    N.check(N.lib().dm_zernike(N.ptr(r), N.ptr(theta), r.numel(), deg.ctypes.data, len(n),
                               N.ptr(out), N.stream_ptr(r.device)), "dm_zernike")
    return out


def zernike(r, theta, n, m, norm=True):
    """Noll-normalised Zernike polynomials Z_n^m(r, theta) on the unit disk, 0
    outside (psf.py:456-548), evaluated by a CUDA kernel in float64 arithmetic.
    ``r``/``theta`` may be CUDA tensors (result float32 on the device) or arrays
    (result a float64 numpy array, stacked over the degrees and squeezed)."""
    if not norm:
        raise ValueError("only the normalised polynomials (norm=True) are provided")
    if isinstance(r, torch.Tensor):
        return _zernike_gpu(r, theta, n, m).squeeze()
    rt = torch.as_tensor(np.asarray(r, np.float64), dtype=torch.float32, device="cuda")
    if not (rt >= 0).all():
        raise ValueError("r must always be greater or equal to 0")
    tt = torch.as_tensor(np.asarray(theta, np.float64), dtype=torch.float32, device="cuda")
    return _zernike_gpu(rt, tt, n, m).squeeze().double().cpu().numpy()


class _PupilDefocus(torch.autograd.Function):
    @staticmethod
    def forward(ctx, p0, kz, zr):
        nx, ny = p0.shape
        nz = zr.numel()
        pupil = torch.empty(nz, nx, ny, dtype=torch.complex64, device=p0.device)
        N.check(N.lib().dm_pupil_defocus(N.ptr(p0), N.ptr(kz), N.ptr(zr), nx, ny, nz,
                                         N.ptr(pupil), N.stream_ptr(p0.device)),
                "dm_pupil_defocus")
        ctx.save_for_backward(p0, kz, zr)
        return pupil

    @staticmethod
    def backward(ctx, g):
        p0, kz, zr = ctx.saved_tensors
        lib = N.lib()
        nx, ny = p0.shape
        nz = zr.numel()
        gp0, gkz, gzr = torch.empty_like(p0), torch.empty_like(kz), torch.empty_like(zr)
        ws = N.WORKSPACES.get("pupil", lib.dm_pupil_defocus_grad_workspace_size(nx, ny, nz),
                              p0.device)
        N.check(lib.dm_pupil_defocus_backward(
            N.ptr(g.contiguous().to(torch.complex64)), N.ptr(p0), N.ptr(kz), N.ptr(zr), nx, ny,
            nz, N.ptr(gp0), N.ptr(gkz), N.ptr(gzr), N.ptr(ws), ws.numel(),
            N.stream_ptr(p0.device)), "dm_pupil_defocus_backward")
        return gp0, gkz, gzr


class _ShiftedIntensity(torch.autograd.Function):
    @staticmethod
    def forward(ctx, field):
        nz, nx, ny = field.shape
        out = torch.empty(nx, ny, nz, dtype=torch.float32, device=field.device)
        N.check(N.lib().dm_shifted_intensity(N.ptr(field), nx, ny, nz, N.ptr(out),
                                             N.stream_ptr(field.device)), "dm_shifted_intensity")
        ctx.save_for_backward(field)
        return out

    @staticmethod
    def backward(ctx, g):
        (field,) = ctx.saved_tensors
        nz, nx, ny = field.shape
        gf = torch.empty_like(field)
        N.check(N.lib().dm_shifted_intensity_backward(
            N.ptr(field), N.ptr(g.contiguous().float()), nx, ny, nz, N.ptr(gf),
            N.stream_ptr(field.device)), "dm_shifted_intensity_backward")
        return gf


class Hanser_psf(nn.Module):
    """Pupil-function PSF with Zernike magnitude and phase aberrations (psf.py:157-371,
    after Hanser et al. 2003/2004 and pyOTF): the aberrated pupil is defocused on
    every z plane, inverse-transformed laterally and squared.  Learnable ``NA``,
    ``wavelength``, ``ni``, ``res_lateral``, ``res_axial``, ``mcoefs``, ``pcoefs``
    (Noll order); ``condition`` "sine" (default), "herschel" or "none";
    ``vec_corr`` is accepted and unused, as in the reference."""

    def __init__(self, box_shape, xi0, xi1, xi2, device="cuda", NA=1.4, wavelength=0.610,
                 ni=1.5, res_lateral=0.1, res_axial=0.25, num_zernike=21, vec_corr="none",
                 condition="sine", with_grad=True):
        super().__init__()
        _cuda_only(device, "Hanser_psf")
        self.with_grad = with_grad
        self.size_x, self.size_y, self.size_z = (int(s) for s in box_shape)
        self.device = device
        mk = self.make_param
        self.NA, self.wavelength, self.ni = mk(NA), mk(wavelength), mk(ni)
        self.res_lateral, self.res_axial = mk(res_lateral), mk(res_axial)
        z = lambda: nn.Parameter(torch.zeros(num_zernike, dtype=torch.float, device=device),
                                 requires_grad=with_grad)
        self.mcoefs, self.pcoefs = z(), z()
        self.xi0, self.xi1, self.xi2 = xi0, xi1, xi2
        self.vec_corr = vec_corr
        if condition not in ("none", "sine", "herschel"):
            raise ValueError(f"unknown condition {condition!r}")
        self.condition = condition
        self._degrees = noll2degrees(np.arange(num_zernike) + 1)

    def make_param(self, x):
        return nn.Parameter(torch.tensor(x, dtype=torch.float, device=self.device),
                            requires_grad=self.with_grad)

    def _gen_zrange(self):
        self.zrange = (torch.arange(self.size_z, device=self.device)
                       - (self.size_z + 1) // 2) * self.res_axial

    def _gen_kr(self):
        kx = torch.fft.fftfreq(self.size_x, dtype=torch.float, device=self.device)
        ky = torch.fft.fftfreq(self.size_y, dtype=torch.float, device=self.device)
        self._kx = kx / self.res_lateral
        self._ky = ky / self.res_lateral
        kxx, kyy = torch.meshgrid(kx, ky, indexing="ij")
        self._phi = torch.atan2(kyy, kxx)
        self._kr = torch.sqrt(kyy ** 2 + kxx ** 2) / self.res_lateral
        self._kmag = self.ni / self.wavelength
        self._kz = torch.sqrt(torch.nn.functional.relu(self._kmag ** 2 - self._kr ** 2))

    def _gen_pupil(self):
        return (self._kr <= self.NA / self.wavelength).type(torch.complex64)

    def _pupil_plane(self, pupil_base):
        """The z-independent factor of the pupil: base times the obliquity factor
        of the sine / Herschel condition (psf.py:337-355)."""
        kr, kmag = self._kr, self._kmag
        theta = torch.arcsin((kr < kmag) * kr / kmag)
        if self.condition == "sine":
            pupil_base = pupil_base * (1.0 / torch.sqrt(torch.cos(theta)))
        elif self.condition == "herschel":
            pupil_base = pupil_base * (1.0 / torch.cos(theta))
        return pupil_base

    def _gen_psf(self, pupil_base=None):
        """Complex field [1, nz, nx, ny] (psf.py:316-365)."""
        self._gen_kr()
        self._gen_zrange()
        if pupil_base is None:
            pupil_base = self._gen_pupil()
        p0 = self._pupil_plane(pupil_base).to(torch.complex64).contiguous()
        pupil = _PupilDefocus.apply(p0, self._kz.contiguous(), self.zrange.float().contiguous())
        field = torch.fft.ifftn(pupil, dim=(1, 2))
        return field.unsqueeze(0)

    def forward(self):
        self._gen_zrange()
        self._gen_kr()
        r = self._kr * self.wavelength / self.NA
        with torch.no_grad():
            zerns = _zernike_gpu(r, self._phi, *self._degrees)
        pupil_phase = (zerns * self.pcoefs[:, None, None]).sum(0)
        pupil_mag = (zerns * self.mcoefs[:, None, None]).sum(0)
        pupil_total = (torch.abs(self._gen_pupil()) + pupil_mag) * torch.exp(1j * pupil_phase)
        field = self._gen_psf(pupil_total)[0]
        return _ShiftedIntensity.apply(field.contiguous())

    def otfi(self, PSFi):
        """Intensity OTF, complex (psf.py:367-370)."""
        return torch.fft.fftshift(torch.fft.fftn(torch.fft.ifftshift(PSFi)))
