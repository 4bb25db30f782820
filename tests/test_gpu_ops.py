"""CUDA narrow band, Gaussian OTF, image-loss, Adam and the fused renderer against
plain PyTorch float32 references of the same operations (the reference's own
expressions) and against the float64 oracle."""
import numpy as np
import pytest
import torch

import oracle
from conftest import rel_l2
from deltamic_b200 import MeshRenderer, ops
from deltamic_b200.mesh import random_sh_shape

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL_CHAIN_V = 2e-4
TOL_CHAIN = 1e-4


def _axes(shape, box):
    return ops.FreqGrid(box, shape).axes(torch.float32, DEV)


def _torch_otf(S, x0, x1, x2):
    g0, g1, g2 = torch.meshgrid(x0, x1, x2, indexing="ij")
    return torch.exp(-(g0 * (S[0, 0] * g0 + S[0, 1] * g1 + S[0, 2] * g2)
                       + g1 * (S[1, 0] * g0 + S[1, 1] * g1 + S[1, 2] * g2)
                       + g2 * (S[2, 0] * g0 + S[2, 1] * g1 + S[2, 2] * g2)) / 2)


@pytest.mark.parametrize("shape", [(16, 16, 16), (33, 20, 17), (64, 64, 64)])
def test_gaussian_otf_and_sigma_grad(shape):
    box = np.array([[-0.4, 0.45]] * 3)
    x = _axes(shape, box)
    S = torch.tensor([[1.0e-3, 2e-4, 0.0], [2e-4, 1.5e-3, 1e-4], [0.0, 1e-4, 2e-3]],
                     device=DEV, requires_grad=True)
    S2 = S.detach().clone().requires_grad_(True)
    otf = ops.gaussian_otf(S, *x)
    ref = _torch_otf(S2, *x)
    assert torch.allclose(otf, ref, rtol=2e-6, atol=1e-30)
    w = torch.randn(shape, device=DEV)
    (otf * w).sum().backward()
    (ref * w).sum().backward()
    assert rel_l2(S.grad.cpu().numpy(), S2.grad.cpu().numpy()) < 1e-4


@pytest.mark.parametrize("thresh", [1e-5, 1e-2, 0.5, 2.0])
def test_narrowband_matches_boolean_mask(thresh):
    box = np.array([[-0.4, 0.45]] * 3)
    x = _axes((70, 64, 50), box)
    otf = ops.gaussian_otf(torch.diag(torch.tensor([1e-3, 2e-3, 4e-3], device=DEV)), *x)
    band = ops.narrowband(otf, thresh)
    ref = torch.nonzero((otf > thresh).reshape(-1)).reshape(-1)
    assert torch.equal(band.long(), ref)


@pytest.mark.parametrize("kind", ["sum", "mse"])
@pytest.mark.parametrize("contrast", [0.0, 0.3])
def test_image_loss_matches_torch_autograd(kind, contrast):
    torch.manual_seed(0)
    shape = (40, 36, 30)
    z = (torch.randn(shape, device=DEV) + 1j * torch.randn(shape, device=DEV)).to(torch.complex64)
    tgt = torch.rand(shape, device=DEV)
    loss, img, gz = ops.image_loss(z, kind, tgt if kind == "mse" else None, contrast,
                                   want_grad=True, want_image=True)
    zr = z.clone().requires_grad_(True)
    a = torch.abs(zr)
    n = ((a - a.min()) / (a.max() - a.min()) + contrast) / (1 + contrast)
    ref = n.sum() if kind == "sum" else torch.mean((n - tgt) ** 2)
    ref.backward()
    assert abs(float(loss) - float(ref)) <= 2e-5 * abs(float(ref))
    assert torch.allclose(img, a.detach(), rtol=1e-6, atol=1e-7)
    assert rel_l2(gz.cpu().numpy(), zr.grad.cpu().numpy()) < 1e-5


def test_image_loss_tied_extrema():
    z = torch.ones(4096, dtype=torch.complex64, device=DEV)
    z[:7] = 0.5
    z[100:103] = 3.0 + 0j
    z[200] = 2.0
    loss, _, gz = ops.image_loss(z, "sum", want_grad=True)
    zr = z.clone().requires_grad_(True)
    a = zr.abs()
    ((a - a.min()) / (a.max() - a.min())).sum().backward()
    assert torch.allclose(gz, zr.grad, rtol=1e-5, atol=1e-6)


def test_adam_matches_torch():
    torch.manual_seed(1)
    p = torch.randn(5000, device=DEV)
    p2 = p.clone().requires_grad_(True)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    step = torch.zeros(1, dtype=torch.int64, device=DEV)
    opt = torch.optim.Adam([p2], lr=1e-3)
    for _ in range(5):
        g = torch.randn_like(p)
        ops.adam_step(p, g, m, v, step, 1e-3)
        p2.grad = g.clone()
        opt.step()
    assert int(step) == 5
    assert torch.allclose(p, p2.detach(), rtol=1e-5, atol=1e-6)


def test_fused_renderer_matches_oracle_pipeline():
    v, f = random_sh_shape(2, 0.3, 4, 0.08, seed=3)
    rng = np.random.default_rng(3)
    c = rng.uniform(0.5, 1.5, len(f))
    box = oracle.compute_box_size(v, 0.2)
    shape = (24, 22, 20)
    sig = np.array([[1.2e-3, 1e-4, 0.0], [1e-4, 1.0e-3, 0.0], [0.0, 0.0, 2e-3]])
    tgt = rng.uniform(0, 1, shape)
    r = MeshRenderer(box, shape, 1e-5, DEV)
    V = torch.tensor(v, dtype=torch.float32, device=DEV, requires_grad=True)
    F = torch.tensor(f, device=DEV)
    C = torch.tensor(c, dtype=torch.float32, device=DEV, requires_grad=True)
    S = torch.tensor(sig, dtype=torch.float32, device=DEV, requires_grad=True)
    T = torch.tensor(tgt, dtype=torch.float32, device=DEV)
    loss = r.loss(V, F, C, "mse", T, sigma=S)
    loss.backward()
    o = oracle.pipeline(v, f, c, box, shape, S.detach().cpu().double().numpy(), 1e-5,
                        loss="mse", target=T.cpu().double().numpy())
    assert abs(r.n_band - len(o["idx"])) <= max(2, len(o["idx"]) // 1000)
    ev = rel_l2(V.grad.cpu().numpy(), o["grad_verts"])
    ec = rel_l2(C.grad.cpu().numpy(), o["grad_coeff"])
    es = rel_l2(S.grad.cpu().numpy(), o["grad_sigma"])
    print("fused renderer vs oracle: loss %.2e verts %.2e coeff %.2e sigma %.2e" % (
        abs(float(loss) - o["loss"]) / abs(o["loss"]), ev, ec, es))
    assert abs(float(loss) - o["loss"]) < 1e-4 * abs(o["loss"])
    # chain tolerance: the larger of a fixed bound and twice the conditioning
    # floor of the float64 gradients (see test_gpu_meshft)
    fl = oracle.chain_floor(v, f, c, box, shape, S.detach().cpu().double().numpy(), 1e-5,
                            "mse", T.cpu().double().numpy())
    print("conditioning floor", fl)
    assert ev < max(TOL_CHAIN_V, 2 * fl["verts"])
    assert ec < max(TOL_CHAIN, 2 * fl["coeff"])
    assert es < max(TOL_CHAIN, 2 * fl["sigma"])
