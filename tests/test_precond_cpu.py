"""Host side of the large-steps preconditioner: the uniform Laplacian against the
published definition of largesteps' compute_matrix (M = I + lambda L, L = D - A
over the mesh edges), its CSR lists, and the Chebyshev plan (interval and
iteration count) through a float64 restatement of the iteration against
(M M)^-1 formed densely."""
import numpy as np
import torch

from deltamic_b200.mesh import icosphere
from deltamic_b200.precond import chebyshev_plan, laplacian_csr, uniform_laplacian


def test_uniform_laplacian_is_degree_minus_adjacency():
    # tetrahedron: every vertex has degree 3 and is adjacent to the three others
    f = np.array([[0, 1, 2], [0, 3, 1], [0, 2, 3], [1, 3, 2]])
    L = uniform_laplacian(f, 4, torch.float64, "cpu").numpy()
    assert np.array_equal(L, 4 * np.eye(4) - np.ones((4, 4)))
    v, f = icosphere(2, 0.3)
    L = uniform_laplacian(f, len(v), torch.float64, "cpu").numpy()
    assert np.allclose(L.sum(1), 0) and np.allclose(L, L.T)
    A = -(L - np.diag(np.diag(L)))
    assert set(np.unique(A)) == {0.0, 1.0}
    assert np.array_equal(np.diag(L), A.sum(1))  # degree 5 or 6 on the icosphere


def test_csr_matches_dense_laplacian():
    v, f = icosphere(3, 0.3)
    nv = len(v)
    rowp, col, deg, edges = laplacian_csr(f, nv, "cpu")
    L = uniform_laplacian(f, nv, torch.float64, "cpu").numpy()
    A = np.zeros((nv, nv))
    rp, cl = rowp.numpy(), col.numpy()
    for i in range(nv):
        row = cl[rp[i]:rp[i + 1]]
        assert np.all(np.diff(row) > 0)
        A[i, row] = 1
    assert np.array_equal(np.diag(L), deg.numpy().astype(float))
    assert np.array_equal(-(L - np.diag(np.diag(L))), A)


def _chebyshev(rowp, col, lam, lo, hi, iters, b):
    """The device iteration restated in float64 (one solve with M)."""
    deg = np.diff(rowp)
    theta, delta = 0.5 * (hi + lo), 0.5 * (hi - lo)

    def M(d):
        s = np.zeros_like(d)
        for i in range(len(deg)):
            s[i] = d[col[rowp[i]:rowp[i + 1]]].sum(0)
        return (1 + lam * deg)[:, None] * d - lam * s

    x = np.zeros_like(b)
    r = b.copy()
    d = r / theta
    rho = delta / theta
    for _ in range(iters):
        rho1 = 1.0 / (2.0 * theta / delta - rho)
        x = x + d
        r = r - M(d)
        d = rho1 * rho * d + (2.0 * rho1 / delta) * r
        rho = rho1
    return x


def test_chebyshev_plan_reaches_its_tolerance():
    v, f = icosphere(2, 0.3)
    nv = len(v)
    rowp, col, deg, edges = laplacian_csr(f, nv, "cpu")
    L = uniform_laplacian(f, nv, torch.float64, "cpu").numpy()
    ev = np.linalg.eigvalsh(L)
    rng = np.random.default_rng(0)
    g = rng.normal(size=(nv, 3))
    for lam in (5.0, 20.0, 50.0):
        lo, hi, iters = chebyshev_plan(deg, edges, lam, 1e-6)
        assert lo <= 1 + lam * ev[0] + 1e-9 and hi >= 1 + lam * ev[-1] - 1e-9
        M = np.eye(nv) + lam * L
        ref = np.linalg.solve(M @ M, g)
        rp, cl = rowp.numpy(), col.numpy()
        y = _chebyshev(rp, cl, lam, lo, hi, iters, g)
        x = _chebyshev(rp, cl, lam, lo, hi, iters, y)
        err = np.linalg.norm(x - ref) / np.linalg.norm(ref)
        assert err < 2e-6, (lam, iters, err)
