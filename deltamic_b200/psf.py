"""Gaussian OTF generators of deltaMic (``deltamic/psf.py:8-20``) on the B200 kernels.

``generate_gaussian_psf(sigma, xi0, xi1, xi2)`` returns ``exp(-(xi^T S xi)/2)`` on
the outer grid of the axes, differentiable in ``sigma`` (a [3,3] CUDA tensor);
``generate_gaussian_psf_from_sigma`` is the isotropic form ``exp(-s |xi|^2 / 2)``.
"""
from __future__ import annotations

import torch

from . import ops

__all__ = ["generate_gaussian_psf", "generate_gaussian_psf_from_sigma"]


def generate_gaussian_psf(sigma, xi0, xi1, xi2):
    """exp(-(xi^T sigma xi)/2) on the grid of the axes (float32 kernel; a float64
    sigma or float64 axes give a float64 result with gradients to sigma)."""
    if sigma.dtype == torch.float64 or xi0.dtype == torch.float64:
        return ops.gaussian_otf(sigma.float(), xi0, xi1, xi2).double()
    return ops.gaussian_otf(sigma, xi0, xi1, xi2)


def generate_gaussian_psf_from_sigma(sigma, xi0, xi1, xi2):
    s = torch.as_tensor(sigma, dtype=torch.float32, device=xi0.device)
    return ops.gaussian_otf(s * torch.eye(3, device=xi0.device), xi0, xi1, xi2)
