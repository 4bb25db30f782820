"""Batched cells (uneven meshes, grid shapes and PSFs in one launch per stage)
against the single-cell path, cell by cell."""
import numpy as np
import pytest
import torch

import oracle
from conftest import rel_l2
from deltamic_b200 import MeshRenderer
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


def test_batch_matches_single_cells():
    cells = _cells()
    br = BatchRenderer([c[3] for c in cells], [c[4] for c in cells], 1e-5, DEV)
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
        r = MeshRenderer(box, shape, 1e-5, DEV, render_path="dense", autotune=False)
        r.set_sigma(torch.tensor(sig, dtype=torch.float32, device=DEV))
        assert r.n_band == br.band_sizes[i]
        Vi = torch.tensor(v, dtype=torch.float32, device=DEV, requires_grad=True)
        Ci = torch.tensor(c, dtype=torch.float32, device=DEV, requires_grad=True)
        Ti = br.cell_view(target, i).contiguous()
        li = r.loss(Vi, torch.tensor(f, device=DEV), Ci, "mse", Ti)
        li.backward()
        total += float(li)
        assert rel_l2(V.grad[vo[i]:vo[i + 1]].cpu().numpy(), Vi.grad.cpu().numpy()) < 1e-5
        assert rel_l2(C.grad[fo[i]:fo[i + 1]].cpu().numpy(), Ci.grad.cpu().numpy()) < 1e-5
    assert abs(float(loss) - total) < 1e-5 * abs(total)


def test_batch_fit_step_graph_equals_eager():
    cells = _cells(4, seed=3)
    br = BatchRenderer([c[3] for c in cells], [c[4] for c in cells], 1e-5, DEV)
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


def test_batch_cells_match_oracle_pipeline():
    """Every cell of a batch against the float64 oracle chain (meshFT -> render ->
    normalise -> mse -> gradients), with the float32 chain's noise floor."""
    cells = _cells(4, seed=7)
    br = BatchRenderer([c[3] for c in cells], [c[4] for c in cells], 1e-5, DEV)
    br.set_sigmas([c[5] for c in cells])
    br.set_meshes([c[0] for c in cells], [c[1] for c in cells])
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
