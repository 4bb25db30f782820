"""Preconditioned fit step on the GPU against the oracle: the large-steps operator
(M M)^-1, its HBM-bound application, VectorAdam, and one fit step."""
import numpy as np
import pytest
import torch

import oracle
from conftest import rel_l2
from deltamic_b200 import MeshRenderer
from deltamic_b200.fit import FitStep, mesh_iou, run_fit
from deltamic_b200.mesh import icosphere, random_sh_shape
from deltamic_b200.precond import LargeStepsPreconditioner, vector_adam_step

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.mark.parametrize("level,lam", [(2, 50.0), (3, 10.0)])
def test_operator_and_product_match_oracle(level, lam):
    v, f = icosphere(level, 0.3)
    pc = LargeStepsPreconditioner(torch.tensor(f, device=DEV), len(v), lam, DEV)
    P64 = oracle.fit.precondition_matrix(f, len(v), lam)
    assert pc.ldp % 4 == 0 and pc.ldp >= len(v)
    assert rel_l2(pc.P[:, :len(v)].cpu().numpy(), P64) < 1e-6
    assert float(pc.P[:, len(v):].abs().max() if pc.ldp > len(v) else 0.0) == 0.0
    rng = np.random.default_rng(level)
    g = rng.normal(size=(len(v), 3))
    out = pc.apply(torch.tensor(g, dtype=torch.float32, device=DEV))
    assert rel_l2(out.cpu().numpy(), P64 @ g) < 2e-6


def test_vector_adam_matches_oracle_over_steps():
    rng = np.random.default_rng(1)
    nv = 5000  # multi-block path with the separate step counter
    p = rng.normal(size=(nv, 3))
    P = torch.tensor(p, dtype=torch.float32, device=DEV)
    m = torch.zeros_like(P)
    vv = torch.zeros(nv, dtype=torch.float32, device=DEV)
    t = torch.zeros(1, dtype=torch.int64, device=DEV)
    g1, g2, step = np.zeros((nv, 3)), np.zeros((nv, 3)), 0
    for k in range(4):
        g = rng.normal(size=(nv, 3)) * (k + 1)
        vector_adam_step(P, torch.tensor(g, dtype=torch.float32, device=DEV), m, vv, t, 1e-2)
        p, g1, g2, step = oracle.fit.vector_adam_step(p, g, g1, g2, step, 1e-2)
    assert int(t) == 4
    assert rel_l2(P.cpu().numpy(), p) < 1e-6


def test_preconditioned_fit_step_matches_oracle():
    gt, f = random_sh_shape(2, 0.3, 4, 0.08, seed=2)
    init, _ = icosphere(2, 0.3)
    box = oracle.compute_box_size(np.concatenate([gt, init]), 0.2)
    shape = (32, 32, 32)
    r = MeshRenderer(box, shape, 1e-5, DEV)
    r.set_sigma(torch.diag(torch.tensor([1e-3, 1e-3, 4e-3], device=DEV)))
    F = torch.tensor(f, device=DEV)
    C = torch.ones(len(f), device=DEV)
    img = r.render(torch.tensor(gt, dtype=torch.float32, device=DEV), F, C)
    target = ((img - img.min()) / (img.max() - img.min())).contiguous()
    pc = LargeStepsPreconditioner(F, len(init), 20.0, DEV)
    V = torch.tensor(init, dtype=torch.float32, device=DEV)
    step = FitStep(r, V, F, C, target, "mse", 0.0, 5e-3, graph=False, precond=pc,
                   optimizer="vector_adam")
    step()
    g = step.grad.cpu().numpy().astype(np.float64)  # the step's own vertex gradient
    P64 = oracle.fit.precondition_matrix(f, len(init), 20.0)
    p, _, _, _ = oracle.fit.vector_adam_step(init, P64 @ g, np.zeros_like(init),
                                             np.zeros_like(init), 0, 5e-3)
    assert rel_l2(V.cpu().numpy() - init, p - init) < 1e-4


def _edge_spread(V, f):
    P = V[f]
    e = np.linalg.norm(np.concatenate([P[:, 1] - P[:, 0], P[:, 2] - P[:, 1],
                                       P[:, 0] - P[:, 2]]), axis=1)
    return float(np.quantile(e, 0.99) / np.median(e))


def test_preconditioned_fit_converges_with_regular_edges():
    """At 64^3 the preconditioned fit (VectorAdam on (M M)^-1 g) reaches the target
    shape (IoU >= 0.97, image L2 down 5x) with edge lengths as regular as the
    sphere's; plain Adam is printed alongside."""
    gt, f = random_sh_shape(3, 0.3, 6, 0.08, seed=7)
    init, _ = icosphere(3, 0.3)
    box = oracle.compute_box_size(np.concatenate([gt, init]), 0.2)
    r = MeshRenderer(box, (64, 64, 64), 1e-5, DEV)
    r.set_sigma(torch.diag(torch.tensor([1e-3, 1e-3, 4e-3], device=DEV)))
    F = torch.tensor(f, device=DEV)
    C = torch.ones(len(f), device=DEV)
    G = torch.tensor(gt, dtype=torch.float32, device=DEV)
    img = r.render(G, F, C)
    target = ((img - img.min()) / (img.max() - img.min())).contiguous()
    V0 = torch.tensor(init, dtype=torch.float32, device=DEV)
    plain = run_fit(r, V0, F, C, target, steps=150, lr=1e-3)
    pc = LargeStepsPreconditioner(F, len(init), 20.0, DEV)
    pre = run_fit(r, V0, F, C, target, steps=150, lr=5e-3, precond=pc, optimizer="vector_adam")
    iou_plain = mesh_iou(plain["verts"], G, F, r.grid)
    iou_pre = mesh_iou(pre["verts"], G, F, r.grid)
    sp0 = _edge_spread(init, f)
    sp_plain = _edge_spread(plain["verts"].cpu().numpy(), f)
    sp_pre = _edge_spread(pre["verts"].cpu().numpy(), f)
    print(f"IoU plain {iou_plain:.4f} preconditioned {iou_pre:.4f}; image L2 "
          f"{float(pre['losses'][0]):.2e} -> plain {float(plain['losses'][-1]):.2e} / "
          f"preconditioned {float(pre['losses'][-1]):.2e}; edge p99/median sphere {sp0:.2f} "
          f"plain {sp_plain:.2f} preconditioned {sp_pre:.2f}")
    assert iou_pre >= 0.97
    assert float(pre["losses"][-1]) < 0.2 * float(pre["losses"][0])
    assert sp_pre < 1.5 * sp0


@pytest.mark.parametrize("level,lam", [(3, 20.0), (5, 50.0)])
def test_chebyshev_form_matches_oracle_operator(level, lam):
    """The sparse form (two Chebyshev solves with M, no formed operator) against the
    oracle's (M M)^-1 and against the dense form, and under a CUDA graph."""
    v, f = icosphere(level, 0.3)
    F = torch.tensor(f, device=DEV)
    pc = LargeStepsPreconditioner(F, len(v), lam, DEV, method="chebyshev")
    assert pc.method == "chebyshev" and pc.P is None
    rng = np.random.default_rng(level)
    g = rng.normal(size=(len(v), 3))
    G = torch.tensor(g, dtype=torch.float32, device=DEV)
    out = pc.apply(G)
    dense = LargeStepsPreconditioner(F, len(v), lam, DEV, method="dense").apply(G)
    if level <= 3:
        P64 = oracle.fit.precondition_matrix(f, len(v), lam)
        assert rel_l2(out.cpu().numpy(), P64 @ g) < 1e-5
    assert rel_l2(out.cpu().numpy(), dense.cpu().numpy()) < 1e-5
    print(f"level {level} lambda {lam}: {pc.iters} iterations per solve, interval "
          f"[{pc.lo}, {pc.hi}]")
    # graph replay gives the eager result
    o2 = torch.empty_like(G)
    side = torch.cuda.Stream(device=DEV)
    side.wait_stream(torch.cuda.current_stream(DEV))
    with torch.cuda.stream(side):
        pc.apply(G, o2)
    torch.cuda.current_stream(DEV).wait_stream(side)
    gr = torch.cuda.CUDAGraph()
    with torch.cuda.graph(gr):
        pc.apply(G, o2)
    o2.zero_()
    gr.replay()
    torch.cuda.synchronize()
    assert torch.equal(o2, out)
