"""Batched cells (uneven meshes, grid shapes and PSFs in one launch per stage)
against the single-cell path and against the float64 oracle chain, cell by cell,
on both render paths (band-box DFTs of all cells per launch; batched cuFFT)."""
import numpy as np
import pytest
import torch

import oracle
from conftest import rel_l2
from deltamic_b200 import MeshRenderer, ops
from deltamic_b200.batch import BatchFitStep, BatchRenderer
from deltamic_b200.mesh import random_sh_shape

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _cells(n=5, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        level = int(rng.integers(1, 4))
        shape = [(24, 24, 24), (32, 32, 32), (20, 28, 24)][i % 3]
        v, f = random_sh_shape(level, 0.3, 4, 0.08, seed=100 + i)
        box = oracle.compute_box_size(v, 0.2)
        sig = np.diag(rng.uniform(5e-4, 4e-3, 3))
        c = rng.uniform(0.5, 1.5, len(f))
        out.append((v, f, c, box, shape, sig))
    return out


@pytest.mark.parametrize("path", ["dense", "bandbox"])
def test_batch_matches_single_cells(path):
    cells = _cells()
    br = BatchRenderer([c[3] for c in cells], [c[4] for c in cells], 1e-5, DEV,
                       render_path=path)
    br.set_sigmas([c[5] for c in cells])
    br.set_meshes([c[0] for c in cells], [c[1] for c in cells])
    V = torch.tensor(np.concatenate([c[0] for c in cells]), dtype=torch.float32, device=DEV,
                     requires_grad=True)
    C = torch.tensor(np.concatenate([c[2] for c in cells]), dtype=torch.float32, device=DEV,
                     requires_grad=True)
    rng = np.random.default_rng(1)
    target = torch.tensor(rng.uniform(0, 1, br.grid_elems), dtype=torch.float32, device=DEV)
    loss = br.loss(V, C, "mse", target)
    loss.backward()

    vo = np.cumsum([0] + [len(c[0]) for c in cells])
    fo = np.cumsum([0] + [len(c[1]) for c in cells])
    total = 0.0
    for i, (v, f, c, box, shape, sig) in enumerate(cells):
        # the batch renders through cuFFT: compare with the single cell's dense path,
        # on the tile variants the batch was planned with (a different variant sums
        # in another order, and the normalised loss's gradient amplifies rounding at
        # the image minimum, where |z| is near zero)
        r = MeshRenderer(box, shape, 1e-5, DEV, render_path=path, autotune=False)
        r.set_sigma(torch.tensor(sig, dtype=torch.float32, device=DEV))
        assert r.n_band == br.band_sizes[i]
        assert r.use_bandbox == (path == "bandbox") and br.use_bandbox == (path == "bandbox")
        Vi = torch.tensor(v, dtype=torch.float32, device=DEV, requires_grad=True)
        Ci = torch.tensor(c, dtype=torch.float32, device=DEV, requires_grad=True)
        Ti = br.cell_view(target, i).contiguous()
        li = r.loss(Vi, torch.tensor(f, device=DEV), Ci, "mse", Ti)
        li.backward()
        total += float(li)
        assert rel_l2(V.grad[vo[i]:vo[i + 1]].cpu().numpy(), Vi.grad.cpu().numpy()) < 1e-5
        assert rel_l2(C.grad[fo[i]:fo[i + 1]].cpu().numpy(), Ci.grad.cpu().numpy()) < 1e-5
    assert abs(float(loss) - total) < 1e-5 * abs(total)
    assert br.device_error() == 0


@pytest.mark.parametrize("path", ["dense", "bandbox"])
def test_batch_fit_step_graph_equals_eager(path):
    cells = _cells(4, seed=3)
    br = BatchRenderer([c[3] for c in cells], [c[4] for c in cells], 1e-5, DEV,
                       render_path=path)
    br.set_sigmas([c[5] for c in cells])
    br.set_meshes([c[0] for c in cells], [c[1] for c in cells])
    V0 = torch.tensor(np.concatenate([c[0] for c in cells]), dtype=torch.float32, device=DEV)
    C = torch.tensor(np.concatenate([c[2] for c in cells]), dtype=torch.float32, device=DEV)
    target = torch.rand(br.grid_elems, device=DEV)
    a = BatchFitStep(br, V0.clone(), C, target, graph=True)
    b = BatchFitStep(br, V0.clone(), C, target, graph=False)
    for _ in range(3):
        la, lb = float(a()[0]), float(b()[0])
        assert abs(la - lb) <= 1e-6 * abs(lb)
    assert torch.equal(a.V, b.V)


@pytest.mark.parametrize("path", ["dense", "bandbox"])
def test_batch_cells_match_oracle_pipeline(path):
    """Every cell of a batch against the float64 oracle chain (meshFT -> render ->
    normalise -> mse -> gradients), with the float32 chain's noise floor."""
    cells = _cells(4, seed=7)
    br = BatchRenderer([c[3] for c in cells], [c[4] for c in cells], 1e-5, DEV,
                       render_path=path)
    br.set_sigmas([c[5] for c in cells])
    br.set_meshes([c[0] for c in cells], [c[1] for c in cells])
    assert br.use_bandbox == (path == "bandbox")
    V = torch.tensor(np.concatenate([c[0] for c in cells]), dtype=torch.float32, device=DEV,
                     requires_grad=True)
    C = torch.tensor(np.concatenate([c[2] for c in cells]), dtype=torch.float32, device=DEV,
                     requires_grad=True)
    rng = np.random.default_rng(8)
    target = torch.tensor(rng.uniform(0, 1, br.grid_elems), dtype=torch.float32, device=DEV)
    loss = br.loss(V, C, "mse", target)
    loss.backward()
    vo = np.cumsum([0] + [len(c[0]) for c in cells])
    fo = np.cumsum([0] + [len(c[1]) for c in cells])
    total = 0.0
    for i, (v, f, c, box, shape, sig) in enumerate(cells):
        t64 = br.cell_view(target, i).cpu().double().numpy()
        o = oracle.pipeline(v, f, c, box, shape, sig, 1e-5, loss="mse", target=t64)
        fl = oracle.chain_floor(v, f, c, box, shape, sig, 1e-5, "mse", t64)
        total += o["loss"]
        ev = rel_l2(V.grad[vo[i]:vo[i + 1]].cpu().numpy(), o["grad_verts"])
        ec = rel_l2(C.grad[fo[i]:fo[i + 1]].cpu().numpy(), o["grad_coeff"])
        print(f"cell {i} {shape}: verts {ev:.2e} coeff {ec:.2e} floor {fl}")
        assert ev < max(2e-4, 2 * fl["verts"])
        assert ec < max(1e-4, 2 * fl["coeff"])
    assert abs(float(loss) - total) < 1e-4 * abs(total)


def test_batch_bandbox_wide_bands_and_image():
    """Cells whose band extent along the line axis needs the two-chunk gradient
    pass (above 32), mixed with narrow ones and three grid shapes: image, per-cell
    loss and dL/dS of the batched band-box DFTs against the batched cuFFT chain on
    the same spectra.  One dominant frequency per cell keeps |z| away from zero,
    so the normalised loss's gradient at the image minimum is well determined."""
    rng = np.random.default_rng(11)
    cells = []
    for i, (shape, sz) in enumerate([((40, 36, 80), 5e-4), ((32, 32, 32), 2e-3),
                                     ((48, 40, 64), 6e-4)]):
        v, f = random_sh_shape(2, 0.3, 4, 0.08, seed=200 + i)
        box = oracle.compute_box_size(v, 0.2)
        cells.append((v, f, rng.uniform(0.5, 1.5, len(f)), box, shape,
                      np.diag([2e-3, 2e-3, sz])))
    rs = {}
    for path in ("dense", "bandbox"):
        br = BatchRenderer([c[3] for c in cells], [c[4] for c in cells], 1e-5, DEV,
                           render_path=path)
        br.set_sigmas([c[5] for c in cells])
        br.set_meshes([c[0] for c in cells], [c[1] for c in cells])
        assert br.use_bandbox == (path == "bandbox")
        rs[path] = br
    bb, dn = rs["bandbox"], rs["dense"]
    V = torch.tensor(np.concatenate([c[0] for c in cells]), dtype=torch.float32, device=DEV)
    C = torch.tensor(np.concatenate([c[2] for c in cells]), dtype=torch.float32, device=DEV)
    ft = bb.forward_spectrum(V, C, dense=False)
    offs = np.concatenate([[0], np.cumsum(bb.band_sizes)])
    band = bb.band.long()
    gidx = torch.cat([band[offs[i]:offs[i + 1]] + bb.grid_offset[i] for i in range(len(cells))])
    otf_b = bb.otf[gidx]
    for i in range(len(cells)):  # one dominant frequency per cell
        sl = slice(int(offs[i]), int(offs[i + 1]))
        o = otf_b[sl]
        k = int(torch.argmax(o))
        ft[sl] = 0.3 * ft[sl] / float((ft[sl].abs() * o).sum())
        ft[sl][k] += 1.0 / float(o[k])
    # the cuFFT chain on the same spectra
    dn.spec.zero_()
    dn.spec[gidx] = ft * otf_b
    dn.inverse_fft()
    _, img0, _ = dn.image_loss("sum", None, want_grad=False, want_image=True)
    target = torch.empty_like(img0)
    for i in range(len(cells)):
        x = dn.cell_view(img0, i)
        nx = (x - x.min()) / (x.max() - x.min())
        noise = torch.tensor(rng.normal(size=x.shape), dtype=torch.float32, device=DEV)
        dn.cell_view(target, i).copy_(nx + 0.05 * noise)
    ld, imgd, gz = dn.image_loss("mse", target, want_grad=True, want_image=True)
    dn.adjoint_fft(gz)
    Gd = dn.G[gidx]
    lb, Gb, imgb = bb.render_loss_bandbox(ft, "mse", target, want_grad=True, want_image=True)
    torch.cuda.synchronize()
    assert bb.device_error() == 0
    for i in range(len(cells)):
        sl = slice(int(offs[i]), int(offs[i + 1]))
        e_img = rel_l2(bb.cell_view(imgb, i).cpu().numpy(), dn.cell_view(imgd, i).cpu().numpy())
        e_l = abs(float(lb[i]) - float(ld[i])) / abs(float(ld[i]))
        # the same cell through the single-box call: the batch repeats its arithmetic
        band_i = bb.band[sl].contiguous()
        plan = ops.BandBox(bb.grids[i], band_i)
        _, _, G1 = ops.render_loss_bandbox(ft[sl].contiguous(), band_i, plan,
                                           bb.cell_view(bb.otf, i).contiguous(), "mse",
                                           bb.cell_view(target, i).contiguous())
        e_b1 = rel_l2(Gb[sl].cpu().numpy(), (G1 / bb.grids[i].numel).cpu().numpy())
        # dL/dS in float64 from the same float32 spectrum and target
        idx = band_i.cpu().numpy().astype(np.int64)
        otf64 = bb.cell_view(bb.otf, i).cpu().double().numpy()
        t64 = bb.cell_view(target, i).cpu().double().numpy()
        img64, z64 = oracle.render_from_band(ft[sl].cpu().numpy().astype(np.complex128), idx,
                                             otf64)
        gimg = oracle.image_loss_backward(img64, "mse", t64)
        gz = np.where(np.abs(z64) > 0, gimg * z64 / np.abs(z64), 0.0)
        G64 = (np.fft.fftn(gz) / gz.size).ravel()[idx]
        eb = rel_l2(Gb[sl].cpu().numpy(), G64)
        ed = rel_l2(Gd[sl].cpu().numpy(), G64)
        print(f"cell {i} {cells[i][4]} extent {plan.extent}: image {e_img:.2e} loss {e_l:.2e}; "
              f"dL/dS vs float64: band-box batch {eb:.2e} (single box {e_b1:.2e} apart), "
              f"cuFFT chain {ed:.2e}")
        assert e_img < 2e-6 and e_l < 5e-5, i
        assert e_b1 < 1e-6, i
        assert eb < max(2e-5, 3 * ed), i
