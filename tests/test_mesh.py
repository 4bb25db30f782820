"""Synthetic mesh generators."""
import numpy as np
import pytest

from deltamic_b200.mesh import icosphere, random_sh_shape, sh_perturb


@pytest.mark.parametrize("level,nv,nt", [(0, 12, 20), (2, 162, 320), (3, 642, 1280),
                                         (4, 2562, 5120), (5, 10242, 20480)])
def test_icosphere_counts_and_closure(level, nv, nt):
    v, f = icosphere(level, 0.3)
    assert v.shape == (nv, 3) and f.shape == (nt, 3)
    assert np.allclose(np.linalg.norm(v, axis=1), 0.3)
    edges = np.sort(np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]]), axis=1)
    ne = len(np.unique(edges, axis=0))
    assert nv - ne + nt == 2          # closed genus-0 surface
    p = v[f]
    n = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    assert np.all(np.einsum("ij,ij->i", n, p.mean(axis=1)) > 0)  # outward


def test_sh_shape_is_seeded():
    a, fa = random_sh_shape(3, 0.3, 6, 0.08, seed=7)
    b, fb = random_sh_shape(3, 0.3, 6, 0.08, seed=7)
    c, _ = random_sh_shape(3, 0.3, 6, 0.08, seed=8)
    assert np.array_equal(a, b) and np.array_equal(fa, fb) and not np.array_equal(a, c)


def test_real_sph_harm_orthonormal():
    from deltamic_b200.mesh import real_sph_harm
    rng = np.random.default_rng(0)
    x = rng.normal(size=(200000, 3))
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    th, ph = np.arccos(x[:, 2]), np.arctan2(x[:, 1], x[:, 0])
    ys = [real_sph_harm(l, m, th, ph) for l in range(0, 4) for m in range(-l, l + 1)]
    G = np.array([[np.mean(a * b) * 4 * np.pi for b in ys] for a in ys])
    assert np.allclose(G, np.eye(len(ys)), atol=3e-2)
