"""Reference entry points under their own names: ``MeshFTCUDA.apply``
(cuda_class.py:10-41) against the float64 oracle on raw vertex coordinates,
``compute_precondition_matrix`` and ``VectorAdam`` (optimize.py:207-258) against
the oracle's operator and update.  Tolerances as the meshFT tests: spectrum 1e-5,
vertex gradient 1e-4 (rel-L2, float32 kernels vs float64); operator 1e-6 (it is
formed in float64); VectorAdam over four steps 1e-6."""
import numpy as np
import pytest
import torch

import oracle
from conftest import rel_l2
from deltamic_b200.cuda_class import MeshFTCUDA
from deltamic_b200.mesh import icosphere, random_sh_shape
from deltamic_b200.optimize import VectorAdam, compute_precondition_matrix
from deltamic_b200.render import (compute_box_size, compute_spatial_frequency_grid,
                                  get_internal_triangle_and_mesh_areas_with_coeff)
from deltamic_b200.psf import generate_gaussian_psf

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.mark.parametrize("shape", [(24, 20, 18), (25, 25, 25)])
def test_meshftcuda_matches_oracle_on_raw_coordinates(shape):
    v, f = random_sh_shape(2, 0.3, 4, 0.08, 3)
    v = v + np.array([0.05, -0.12, 0.2])  # coordinates as given: no box shift
    c = np.random.default_rng(4).uniform(0.5, 1.5, len(f))
    box = compute_box_size(v, 0.2)
    xi0, xi1, xi2 = compute_spatial_frequency_grid(shape, box[:, 1] - box[:, 0], device=DEV)
    otf = generate_gaussian_psf(torch.diag(torch.tensor([1e-3, 1e-3, 4e-3], device=DEV)),
                                xi0, xi1, xi2)
    V = torch.tensor(v, dtype=torch.float32, device=DEV, requires_grad=True)
    F = torch.tensor(f, device=DEV)
    C = torch.tensor(c, dtype=torch.float32, device=DEV, requires_grad=True)
    ft = MeshFTCUDA.apply(V, F, C, xi0, xi1, xi2, otf, 1e-5)
    assert ft.shape == shape and ft.dtype == torch.complex64
    mask = (otf > 1e-5).cpu().numpy()
    axes = [x.double().cpu().numpy() for x in (xi0, xi1, xi2)]
    g0, g1, g2 = np.meshgrid(*axes, indexing="ij")
    xil = np.stack([g0[mask], g1[mask], g2[mask]], axis=1)
    ref = oracle.meshft_forward(v, f, c, xil)
    got = ft.detach().cpu().numpy()
    assert rel_l2(got[mask], ref) < 1e-5
    assert np.all(got[~mask] == 0)
    rng = np.random.default_rng(6)
    G = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    Gt = torch.tensor(G, dtype=torch.complex64, device=DEV)
    (ft * Gt.conj()).real.sum().backward()
    rv, _ = oracle.meshft_backward(v, f, c, xil, G[mask].astype(np.complex64), ref)
    assert rel_l2(V.grad.cpu().numpy(), rv) < 1e-4
    assert C.grad is None  # the reference returns no coefficient gradient


def test_area_helper_with_coeff():
    v, f = icosphere(2, 0.3)
    c = np.random.default_rng(1).uniform(0.5, 1.5, len(f))
    trisar, meshar = get_internal_triangle_and_mesh_areas_with_coeff(
        torch.tensor(v, device=DEV), torch.tensor(f, device=DEV), torch.tensor(c, device=DEV))
    t = v[f]
    a = 0.5 * np.linalg.norm(np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]), axis=1)
    assert rel_l2(trisar.cpu().numpy(), c * a) < 1e-12
    assert abs(float(meshar) - float((c * a).sum())) < 1e-12


def test_compute_precondition_matrix_and_vector_adam():
    v, f = icosphere(2, 0.3)
    V = torch.tensor(v, dtype=torch.float32, device=DEV)
    P = compute_precondition_matrix(V, torch.tensor(f, device=DEV), 20.0)
    assert P.dtype == torch.float32 and P.shape == (len(v), len(v))
    assert rel_l2(P.cpu().numpy(), oracle.fit.precondition_matrix(f, len(v), 20.0)) < 1e-6

    rng = np.random.default_rng(2)
    p = rng.normal(size=(len(v), 3))
    param = torch.nn.Parameter(torch.tensor(p, dtype=torch.float32, device=DEV))
    opt = VectorAdam([param], lr=1e-2)
    g1, g2, step = np.zeros_like(p), np.zeros_like(p), 0
    for k in range(4):
        g = rng.normal(size=p.shape) * (k + 1)
        param.grad = torch.tensor(g, dtype=torch.float32, device=DEV)
        opt.step()
        p, g1, g2, step = oracle.fit.vector_adam_step(p, g, g1, g2, step, 1e-2)
    assert rel_l2(param.detach().cpu().numpy(), p) < 1e-6

    # axis=None: elementwise Adam (torch.optim.Adam's update)
    q = torch.nn.Parameter(torch.tensor(rng.normal(size=(7, 5)), dtype=torch.float32,
                                        device=DEV))
    q_ref = torch.nn.Parameter(q.detach().clone())
    opt_q = VectorAdam([q], lr=1e-2, axis=None)
    opt_ref = torch.optim.Adam([q_ref], lr=1e-2)
    for _ in range(3):
        g = torch.randn(7, 5, device=DEV)
        q.grad, q_ref.grad = g.clone(), g.clone()
        opt_q.step()
        opt_ref.step()
    assert rel_l2(q.detach().cpu().numpy(), q_ref.detach().cpu().numpy()) < 1e-6
