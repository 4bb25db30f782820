"""Oracle of the preconditioned fit step: known answers for the uniform Laplacian,
the large-steps operator and VectorAdam (CPU)."""
import numpy as np

import oracle
from deltamic_b200.mesh import icosphere


def test_uniform_laplacian_known_answers():
    v, f = icosphere(0, 1.0)  # icosahedron: 12 vertices of valence 5, 30 edges
    L = oracle.fit.uniform_laplacian(f, len(v))
    assert np.allclose(np.diag(L), 5.0)
    assert np.allclose(L, L.T)
    assert np.allclose(L.sum(axis=1), 0.0)
    assert int((L < 0).sum()) == 60


def test_precondition_matrix_inverts_m_squared():
    v, f = icosphere(1, 1.0)
    P = oracle.fit.precondition_matrix(f, len(v), 10.0)
    M = np.eye(len(v)) + 10.0 * oracle.fit.uniform_laplacian(f, len(v))
    assert np.allclose(P @ (M @ M), np.eye(len(v)), atol=1e-9)
    # constants are fixed points (L 1 = 0), high frequencies are damped
    assert np.allclose(P @ np.ones(len(v)), 1.0)


def test_vector_adam_first_step_is_lr_along_the_vertex_direction():
    rng = np.random.default_rng(0)
    g = rng.normal(size=(5, 3))
    p, g1, g2, t = oracle.fit.vector_adam_step(np.zeros((5, 3)), g, np.zeros((5, 3)),
                                               np.zeros((5, 3)), 0, 0.1, eps=0.0)
    # first step: m1 = g, m2 = |g|^2 per vertex -> p = -lr g / |g|
    assert t == 1
    assert np.allclose(p, -0.1 * g / np.linalg.norm(g, axis=1, keepdims=True))
