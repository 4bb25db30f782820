"""Spatial Gaussian PSF and OTF-from-PSF stage (the reference notebook's
`OTF = abs(fftshift(fftn(PSF)))`) against plain PyTorch float32 references of the
same operations, and the learnable-PSF gradient through the whole render chain."""
import numpy as np
import pytest
import torch

import oracle
from conftest import rel_l2
from deltamic_b200 import (Fourier3dMesh, Gaussian_psf, MeshRenderer, normalize_tensor,
                           otf_from_psf, render_image_from_ftmesh)
from deltamic_b200.mesh import random_sh_shape

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _torch_psf(S, L, shape):
    ax = [torch.linspace(-L[d] / 2, L[d] / 2, shape[d], device=DEV) for d in range(3)]
    g0, g1, g2 = torch.meshgrid(*ax, indexing="ij")
    return torch.exp(-(g0 * (S[0, 0] * g0 + S[0, 1] * g1 + S[0, 2] * g2)
                       + g1 * (S[1, 0] * g0 + S[1, 1] * g1 + S[1, 2] * g2)
                       + g2 * (S[2, 0] * g0 + S[2, 1] * g1 + S[2, 2] * g2)) / 2)


@pytest.mark.parametrize("shape", [(24, 24, 24), (25, 20, 17)])
def test_gaussian_psf_and_otf_match_torch(shape):
    L = np.array([1.3, 1.1, 0.9])
    sig = torch.tensor([[400.0, 30.0, 0.0], [30.0, 350.0, 20.0], [0.0, 20.0, 600.0]],
                       device=DEV)
    model = Gaussian_psf(shape, L, sigma=1.0, device=DEV)
    with torch.no_grad():
        model.sigma.copy_(sig)
    psf = model()
    S = sig.clone().requires_grad_(True)
    psf_t = _torch_psf(S, L, shape)
    assert rel_l2(psf.detach().cpu().numpy(), psf_t.detach().cpu().numpy()) < 1e-6
    otf = otf_from_psf(psf)
    otf_t = torch.abs(torch.fft.fftshift(torch.fft.fftn(psf_t)))
    assert rel_l2(otf.detach().cpu().numpy(), otf_t.detach().cpu().numpy()) < 1e-6
    g = torch.randn(shape, device=DEV)
    (otf * g).sum().backward()
    (otf_t * g).sum().backward()
    e = rel_l2(model.sigma.grad.cpu().numpy(), S.grad.cpu().numpy())
    print(f"{shape}: sigma grad through abs(fftshift(fftn(PSF))) rel {e:.2e}")
    assert e < 1e-4


def test_learnable_psf_gradient_through_render_chain():
    """d loss / d sigma of a spatial Gaussian PSF through OTF -> band -> render ->
    normalise -> MSE: MeshRenderer.loss(otf=...) against the drop-in chain
    (Fourier3dMesh, render_image_from_ftmesh, normalize_tensor, torch autograd)."""
    v, f = random_sh_shape(2, 0.3, 4, 0.08, seed=4)
    box = oracle.compute_box_size(v, 0.2)
    shape = (24, 24, 24)
    L = box[:, 1] - box[:, 0]
    rng = np.random.default_rng(4)
    target = torch.tensor(rng.uniform(0, 1, shape), dtype=torch.float32, device=DEV)
    V = torch.tensor(v, dtype=torch.float32, device=DEV)
    F = torch.tensor(f, device=DEV)
    C = torch.ones(len(f), device=DEV)
    thresh = 1e-2

    m1 = Gaussian_psf(shape, L, sigma=300.0, device=DEV)
    otf1 = otf_from_psf(m1())
    r = MeshRenderer(box, shape, thresh, DEV)
    loss1 = r.loss(V, F, C, "mse", target, otf=otf1)
    loss1.backward()

    m2 = Gaussian_psf(shape, L, sigma=300.0, device=DEV)
    otf2 = torch.abs(torch.fft.fftshift(torch.fft.fftn(m2())))
    mft = Fourier3dMesh(box, shape, device=DEV, dtype=torch.float32, narrowband_thresh=thresh)
    mft.OTF = otf2.detach()
    img = normalize_tensor(render_image_from_ftmesh(mft(V, F, C), otf2, shape))
    loss2 = torch.mean((img - target) ** 2)
    loss2.backward()
    assert r.n_band == mft.band().numel()
    e_l = abs(float(loss1) - float(loss2)) / float(loss2)
    e_g = rel_l2(m1.sigma.grad.cpu().numpy(), m2.sigma.grad.cpu().numpy())
    print(f"loss rel {e_l:.2e}, sigma grad rel {e_g:.2e}")
    assert e_l < 1e-5
    assert e_g < 2e-3
