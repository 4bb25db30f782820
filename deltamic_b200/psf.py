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
"""
from __future__ import annotations

import numpy as np
import torch
from torch import nn

from . import _native as N
from . import ops

__all__ = ["generate_gaussian_psf", "generate_gaussian_psf_from_sigma", "Gaussian_psf",
           "otf_from_psf"]


def generate_gaussian_psf(sigma, xi0, xi1, xi2):
    """exp(-(xi^T sigma xi)/2) on the grid of the axes (float32 kernel; a float64
    sigma or float64 axes give a float64 result with gradients to sigma)."""
    if sigma.dtype == torch.float64 or xi0.dtype == torch.float64:
        return ops.gaussian_otf(sigma.float(), xi0, xi1, xi2).double()
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
        L = np.asarray(torch.as_tensor(box_size).detach().cpu().double().numpy(), np.float64)
        self.axes = tuple(torch.linspace(-L[d] / 2, L[d] / 2, int(box_shape[d]),
                                         dtype=torch.float32, device=device) for d in range(3))
        self.sigma = nn.Parameter(torch.tensor(np.identity(3) * sigma, dtype=dtype,
                                               device=device), requires_grad=with_grad)

    def forward(self):
        out = ops.gaussian_otf(self.sigma.float(), *self.axes)
        return out.to(self.dtype) if self.dtype != torch.float32 else out


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
