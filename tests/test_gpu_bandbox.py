"""Band-box render (separable DFTs pruned to the narrow band's bounding box, fused
with normalize_tensor and the loss) against the dense chain (cuFFT ifftn, the fused
image-loss kernels, cuFFT fftn) and against float64 references."""
import numpy as np
import pytest
import torch

import oracle
from conftest import rel_l2
from deltamic_b200 import MeshRenderer, ops
from deltamic_b200.fit import FitStep
from deltamic_b200.mesh import icosphere, random_sh_shape

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
ANISO = np.diag([1e-3, 1e-3, 4e-3])
FULL = np.array([[1.2e-3, 1e-4, 0.0], [1e-4, 1.0e-3, 2e-4], [0.0, 2e-4, 3e-3]])
WIDE2 = np.diag([2e-3, 2e-3, 5e-4])
WIDE3 = np.diag([1e-3, 1e-3, 4e-4])


def _case(level, shape, sigma, seed, thresh=1e-5):
    v, f = random_sh_shape(level, 0.3, 4, 0.08, seed=seed)
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.5, 1.5, len(f))
    box = oracle.compute_box_size(v, 0.2)
    grid = ops.FreqGrid(box, shape)
    xi = grid.axes(torch.float32, DEV)
    otf = ops.gaussian_otf(torch.tensor(sigma, dtype=torch.float32, device=DEV), *xi)
    band = ops.narrowband(otf, thresh)
    V = torch.tensor(v, dtype=torch.float32, device=DEV)
    F = torch.tensor(f, device=DEV)
    C = torch.tensor(c, dtype=torch.float32, device=DEV)
    ft = ops.meshft_list(V, F, C, grid, band)
    return grid, otf, band, ft, rng


def _conditioned(ft, band, otf):
    """The normalised render puts part of its gradient on the voxels of the image
    min and max (normalize_tensor), through z/|z| there, which is only as well
    determined as |z|: a mesh render has a minimum of |z| near zero, where z/|z|
    is rounding noise in any float32 evaluation.  One dominant band frequency
    keeps |z| away from zero, so two float32 paths can be compared on G."""
    o = otf.view(-1)[band.long()]
    c = int(torch.argmax(o))
    ft = 0.3 * ft / float((ft.abs() * o).sum())
    ft[c] = ft[c] + 1.0 / float(o[c])
    return ft


def _dense(grid, otf, band, ft, kind, target, contrast):
    spec = torch.zeros(grid.shape, dtype=torch.complex64, device=DEV)
    b = band.long()
    spec.view(-1)[b] = ft * otf.view(-1)[b]
    z = torch.fft.ifftn(spec)
    loss, img, gz = ops.image_loss(z, kind, target, contrast, want_grad=True, want_image=True)
    G = torch.fft.fftn(gz).view(-1)[b]
    return loss, img, G


def _float64_chain(grid, otf, band, ft, kind, target, contrast, z_noise=0.0, seed=0):
    """Loss, image and G = fftn(dL/dz) on the band in float64 from the float32
    spectrum; ``z_noise`` multiplies z by 1 + z_noise * (complex normal noise)."""
    idx = band.cpu().numpy().astype(np.int64)
    S = ft.cpu().numpy().astype(np.complex128) * otf.cpu().numpy().ravel()[idx]
    spec = np.zeros(grid.shape, np.complex128)
    spec.ravel()[idx] = S
    z = np.fft.ifftn(spec)
    if z_noise:
        r = np.random.default_rng(seed)
        z = z * (1.0 + z_noise * (r.normal(size=z.shape) + 1j * r.normal(size=z.shape)))
    img = np.abs(z)
    t64 = None if target is None else target.cpu().numpy().astype(np.float64)
    gimg = oracle.image_loss_backward(img, kind, t64, contrast)
    gz = np.where(img > 0, gimg * z / np.where(img > 0, img, 1.0), 0.0)
    return oracle.image_loss(img, kind, t64, contrast), img, np.fft.fftn(gz).ravel()[idx]


def _g_floor(grid, otf, band, ft, kind, target, contrast, G64):
    """Conditioning of G: its largest relative change when z carries the rounding
    of a float32 transform (relative 1e-7 noise), over two draws."""
    worst = 0.0
    for seed in (1, 2):
        _, _, Gp = _float64_chain(grid, otf, band, ft, kind, target, contrast, 1e-7, seed)
        worst = max(worst, rel_l2(Gp, G64))
    return worst


def test_band_bounds_match_numpy():
    grid, otf, band, _, _ = _case(2, (40, 36, 30), FULL, 1)
    bb = ops.band_bounds(band, grid)
    k = np.stack(np.unravel_index(band.cpu().numpy(), grid.shape), axis=1)
    assert bb == tuple(k.min(0).tolist()) + tuple(k.max(0).tolist())


@pytest.mark.parametrize("level,shape,sigma", [(2, (32, 32, 32), ANISO),
                                               (2, (40, 36, 30), FULL),
                                               (3, (64, 48, 56), ANISO),
                                               (1, (17, 19, 23), FULL),
                                               # band extents along axis 2 of 52 and 58:
                                               # the gradient pass in two chunks
                                               (2, (40, 36, 80), WIDE2),
                                               (3, (64, 64, 96), WIDE3)])
@pytest.mark.parametrize("kind,contrast", [("mse", 0.0), ("mse", 0.25), ("sum", 0.0)])
def test_bandbox_matches_dense_chain(level, shape, sigma, kind, contrast):
    grid, otf, band, ft, rng = _case(level, shape, sigma, 7)
    plan = ops.BandBox(grid, band)
    assert plan.supported
    target = None
    ft = _conditioned(ft, band, otf)
    if kind == "mse":
        # a target near the render keeps the loss gradient well conditioned
        _, img0, _ = _dense(grid, otf, band, ft, "sum", None, 0.0)
        nimg = (img0 - img0.min()) / (img0.max() - img0.min())
        target = (nimg + 0.05 * torch.tensor(rng.normal(size=shape), dtype=torch.float32,
                                             device=DEV)).contiguous()
    ld, imgd, Gd = _dense(grid, otf, band, ft, kind, target, contrast)
    lb, imgb, Gb = ops.render_loss_bandbox(ft, band, plan, otf, kind, target, contrast,
                                           want_grad=True, want_image=True)
    torch.cuda.synchronize()
    e_img = rel_l2(imgb.cpu().numpy(), imgd.cpu().numpy())
    e_loss = abs(float(lb) - float(ld)) / abs(float(ld))
    e_g = rel_l2(Gb.cpu().numpy(), Gd.cpu().numpy())
    _, _, G64 = _float64_chain(grid, otf, band, ft, kind, target, contrast)
    eb, ed = rel_l2(Gb.cpu().numpy(), G64), rel_l2(Gd.cpu().numpy(), G64)
    fl = _g_floor(grid, otf, band, ft, kind, target, contrast, G64)
    print(f"bandbox vs dense {shape} {kind} c={contrast}: image {e_img:.2e} loss {e_loss:.2e} "
          f"G {e_g:.2e}; G vs float64: bandbox {eb:.2e} dense {ed:.2e} floor {fl:.2e}")
    assert e_img < 2e-6
    # the loss is a double sum of float32 residuals (nv - target)^2 on both paths
    assert e_loss < 5e-5
    # G against float64 on the same spectrum: within a small factor of the float32
    # conditioning floor or of the dense cuFFT chain's own error (a target this close
    # to the render leaves a small, noise-driven G that float32 rounding of z moves)
    assert eb < max(2e-5, 3 * fl, 3 * ed)


def test_bandbox_against_float64_dft():
    """z, the loss and G against a float64 restatement of ifftn / fftn on the same
    float32 spectrum."""
    grid, otf, band, ft, rng = _case(2, (24, 22, 20), FULL, 11)
    ft = _conditioned(ft, band, otf)
    plan = ops.BandBox(grid, band)
    target = torch.tensor(rng.uniform(0, 1, grid.shape), dtype=torch.float32, device=DEV)
    lb, imgb, Gb = ops.render_loss_bandbox(ft, band, plan, otf, "mse", target, 0.0,
                                           want_grad=True, want_image=True)
    loss64, img, G64 = _float64_chain(grid, otf, band, ft, "mse", target, 0.0)
    e_img = rel_l2(imgb.cpu().numpy(), img)
    e_g = rel_l2(Gb.cpu().numpy(), G64)
    print(f"bandbox vs float64: image {e_img:.2e} loss {abs(float(lb) - loss64) / loss64:.2e} "
          f"G {e_g:.2e}")
    assert e_img < 1e-6
    assert abs(float(lb) - loss64) < 1e-5 * loss64
    assert e_g < 1e-4


@pytest.mark.parametrize("kind", ["sum", "mse"])
def test_bandbox_tied_extrema(kind):
    """Exactly tied min and max over a quarter of the voxels each: band voxels at
    k2 = 0, n2/4, n2/2, 3n2/4 give z(x) = (A + B i^x2 + C (-1)^x2 + D (-i)^x2)/N,
    exact in the kernels' arithmetic (roots of unity +-1, +-i, integer spectrum).
    The min / max gradients are shared evenly by the tied voxels, as in torch's
    min/max backward."""
    shape = (6, 5, 16)
    grid = ops.FreqGrid([[0.0, 1.0], [0.0, 1.0], [0.0, 1.0]], shape)
    band = torch.tensor([0, 4, 8, 12], dtype=torch.int32, device=DEV)
    plan = ops.BandBox(grid, band)
    assert plan.bounds_tuple == (0, 0, 0, 0, 0, 12)
    S = np.array([3.0 + 1.0j, 2.0 - 1.0j, 1.0, 2.0j])
    ft = torch.tensor(S, dtype=torch.complex64, device=DEV)
    otf = torch.ones(shape, dtype=torch.float32, device=DEV)
    rng = np.random.default_rng(5)
    t64 = rng.uniform(0, 1, shape)
    target = torch.tensor(t64, dtype=torch.float32, device=DEV) if kind == "mse" else None
    lb, imgb, Gb = ops.render_loss_bandbox(ft, band, plan, otf, kind, target, 0.0,
                                           want_grad=True, want_image=True)
    img32 = imgb.cpu().numpy()
    n = np.prod(shape)
    x2 = np.arange(shape[2])
    z = np.broadcast_to((S[0] + S[1] * 1j ** x2 + S[2] * (-1.0) ** x2 + S[3] * (-1j) ** x2) / n,
                        shape).astype(np.complex128)
    img = np.abs(z)
    vals = np.unique(np.round(img * n, 9))
    assert len(vals) == 4 and len(np.unique(img32)) == 4  # 4 levels, each a quarter
    assert (img32 == img32.min()).sum() == n // 4 and (img32 == img32.max()).sum() == n // 4
    gimg = oracle.image_loss_backward(img, kind, t64 if kind == "mse" else None)
    gz = gimg * z / img
    G64 = np.fft.fftn(gz).ravel()[[0, 4, 8, 12]]
    loss64 = oracle.image_loss(img, kind, t64 if kind == "mse" else None)
    print(f"ties {kind}: loss {abs(float(lb) - loss64) / abs(loss64):.2e} "
          f"G {rel_l2(Gb.cpu().numpy(), G64):.2e} |G| {np.abs(G64)}")
    assert abs(float(lb) - loss64) < 1e-5 * abs(loss64)
    assert rel_l2(Gb.cpu().numpy(), G64) < 1e-5


@pytest.mark.parametrize("path", ["dense", "bandbox"])
def test_renderer_paths_match_oracle_pipeline(path):
    v, f = random_sh_shape(2, 0.3, 4, 0.08, seed=3)
    rng = np.random.default_rng(3)
    c = rng.uniform(0.5, 1.5, len(f))
    box = oracle.compute_box_size(v, 0.2)
    shape = (24, 22, 20)
    tgt = rng.uniform(0, 1, shape)
    r = MeshRenderer(box, shape, 1e-5, DEV, render_path=path)
    V = torch.tensor(v, dtype=torch.float32, device=DEV, requires_grad=True)
    F = torch.tensor(f, device=DEV)
    C = torch.tensor(c, dtype=torch.float32, device=DEV, requires_grad=True)
    S = torch.tensor(FULL, dtype=torch.float32, device=DEV, requires_grad=True)
    T = torch.tensor(tgt, dtype=torch.float32, device=DEV)
    loss = r.loss(V, F, C, "mse", T, sigma=S)
    loss.backward()
    assert r.use_bandbox == (path == "bandbox")
    s64 = S.detach().cpu().double().numpy()
    o = oracle.pipeline(v, f, c, box, shape, s64, 1e-5, loss="mse",
                        target=T.cpu().double().numpy())
    fl = oracle.chain_floor(v, f, c, box, shape, s64, 1e-5, "mse", T.cpu().double().numpy())
    ev = rel_l2(V.grad.cpu().numpy(), o["grad_verts"])
    ec = rel_l2(C.grad.cpu().numpy(), o["grad_coeff"])
    es = rel_l2(S.grad.cpu().numpy(), o["grad_sigma"])
    print(f"{path}: loss {abs(float(loss) - o['loss']) / o['loss']:.2e} verts {ev:.2e} "
          f"coeff {ec:.2e} sigma {es:.2e} floor {fl}")
    assert abs(float(loss) - o["loss"]) < 1e-4 * abs(o["loss"])
    assert ev < max(2e-4, 2 * fl["verts"])
    assert ec < max(1e-4, 2 * fl["coeff"])
    assert es < max(1e-4, 2 * fl["sigma"])


def test_fit_step_paths_agree_200cube():
    """The 200^3 fit step (level-5 meshes, 20,480 faces): band-box and dense paths
    give the same loss trajectory, and the band-box graph replays its eager step."""
    gt, faces = random_sh_shape(5, 0.3, 6, 0.08, seed=1234)
    init, _ = icosphere(5, 0.3)
    box = oracle.compute_box_size(np.concatenate([gt, init]), 0.2)
    shape = (200, 200, 200)
    F = torch.tensor(faces, device=DEV)
    C = torch.ones(len(faces), device=DEV)
    losses = {}
    for path in ("dense", "bandbox"):
        r = MeshRenderer(box, shape, 1e-5, DEV, render_path=path)
        r.set_sigma(torch.diag(torch.tensor([1e-3, 1e-3, 4e-3], device=DEV)))
        img = r.render(torch.tensor(gt, dtype=torch.float32, device=DEV), F, C)
        target = ((img - img.min()) / (img.max() - img.min())).contiguous()
        if path == "bandbox":
            assert r.use_bandbox and max(r.bbox.extent) <= 64
        V = torch.tensor(init, dtype=torch.float32, device=DEV)
        step = FitStep(r, V, F, C, target, "mse", 0.0, 1e-3, graph=True)
        out = []
        for _ in range(5):
            step()
            out.append(float(step.loss[0]))
        losses[path] = np.array(out)
    print("losses", losses)
    assert np.max(np.abs(losses["bandbox"] - losses["dense"]) / losses["dense"]) < 1e-4

