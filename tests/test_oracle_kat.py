"""Known-answer and finite-difference checks of the oracle (float64)."""
import numpy as np
import pytest

import oracle
from deltamic_b200.mesh import icosphere, jitter, sh_perturb


def _small_case(seed=0, level=1, shape=(15, 15, 15)):
    rng = np.random.default_rng(seed)
    v, f = icosphere(level, 0.3)
    v = jitter(v, 0.01, rng)
    c = rng.uniform(0.5, 1.5, len(f))
    box = oracle.compute_box_size(v, 0.2)
    return v, f, c, box, shape


def test_ft_at_zero_frequency_is_one():
    v, f, c, box, shape = _small_case(shape=(9, 9, 9))
    xi = np.zeros((1, 3))
    ft = oracle.meshft_forward(v - box[:, 0], f, c, xi)
    assert abs(ft[0] - 1.0) < 1e-14


def test_translation_is_a_phase():
    v, f, c, box, shape = _small_case()
    axes = oracle.frequency_axes(box, shape)
    idx = np.arange(0, np.prod(shape), 7)
    xi = oracle.xi_list_from_band(idx, axes)
    t = np.array([0.013, -0.021, 0.007])
    ft0 = oracle.meshft_forward(v, f, c, xi)
    ft1 = oracle.meshft_forward(v + t, f, c, xi)
    assert np.allclose(ft1, ft0 * np.exp(-1j * xi @ t), rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("shape", [(15, 15, 15), (16, 13, 12)])
def test_hermitian_band_and_spectrum(shape):
    """The two facts behind evaluating half of a symmetric band: a Gaussian OTF's
    band is closed under xi -> -xi, which on the centred grid maps flat voxel
    index i to N-1-i, and the mesh transform obeys ft(-xi) = conj(ft(xi))."""
    v, f, c, box, _ = _small_case(seed=3)
    axes = oracle.frequency_axes(box, shape)
    sigma = np.array([[2e-3, 4e-4, 0.0], [4e-4, 1e-3, -3e-4], [0.0, -3e-4, 4e-3]])
    otf = oracle.gaussian_otf(sigma, *axes)
    band = oracle.band_indices(otf, 1e-5)
    n = int(np.prod(shape))
    assert np.array_equal(band[::-1], n - 1 - band)
    xi = oracle.xi_list_from_band(band, axes)
    assert np.array_equal(xi[::-1], -xi)
    ft = oracle.meshft_forward(v - box[:, 0], f, c, xi)
    assert np.allclose(ft[::-1], np.conj(ft), rtol=0, atol=1e-13)


def test_coefficient_scale_invariance():
    v, f, c, box, shape = _small_case()
    o = oracle.pipeline(v, f, c, box, shape, 1e-3 * np.eye(3), 1e-5, loss="sum")
    assert abs(np.dot(c, o["grad_coeff"])) < 1e-9 * np.abs(o["grad_coeff"]).sum()


def test_sphere_shell_transform():
    """A fine icosphere approaches the sphere-shell transform sin(kR)/(kR)."""
    v, f = icosphere(5, 1.0)
    ks = np.array([0.5, 1.5, 3.0, 6.0])
    xi = np.stack([ks * 0.6, ks * 0.0, ks * 0.8], axis=1)
    ft = oracle.meshft_forward(v, f, np.ones(len(f)), xi)
    ana = np.sin(ks) / ks
    assert np.max(np.abs(ft - ana)) < 2e-3


@pytest.mark.parametrize("which", ["verts", "coeff"])
def test_oracle_adjoint_matches_finite_differences(which):
    """FD of the linear functional L = Re sum conj(g) ft(V, c) for a fixed random g:
    its exact gradient is meshft_backward(g) (no min/max kinks involved)."""
    v, f, c, box, shape = _small_case(seed=3, shape=(12, 12, 12))
    rng = np.random.default_rng(5)
    axes = oracle.frequency_axes(box, shape)
    xi = oracle.xi_list_from_band(np.arange(np.prod(shape)), axes)
    vs = v - box[:, 0]
    g = rng.normal(size=len(xi)) + 1j * rng.normal(size=len(xi))
    ft = oracle.meshft_forward(vs, f, c, xi)
    gv, gc = oracle.meshft_backward(vs, f, c, xi, g, ft)

    def L(vv, cc):
        return float(np.real(np.sum(np.conj(g) * oracle.meshft_forward(vv, f, cc, xi))))

    h = 1e-6
    if which == "verts":
        d = rng.normal(size=v.shape)
        fd = (L(vs + h * d, c) - L(vs - h * d, c)) / (2 * h)
        an = np.sum(gv * d)
        # float64 cancellation in near-degenerate pairs limits the FD itself
        tol = 3e-5
    else:
        d = rng.normal(size=c.shape)
        fd = (L(vs, c + h * d) - L(vs, c - h * d)) / (2 * h)
        an = np.sum(gc * d)
        tol = 1e-9
    assert abs(fd - an) <= tol * abs(an), (fd, an)


def test_oracle_sigma_gradient_matches_finite_differences():
    v, f, c, box, shape = _small_case(seed=3, shape=(12, 12, 12))
    sig = np.array([[1.2e-3, 1e-4, 0.0], [1e-4, 1.0e-3, 0.0], [0.0, 0.0, 2e-3]])
    base = oracle.pipeline(v, f, c, box, shape, sig, 1e-5, loss="sum")
    d = np.array([[1.0, 0.3, 0.0], [0.3, 0.5, 0.0], [0.0, 0.0, -0.7]])
    h = 1e-9

    def L(s):
        return oracle.pipeline(v, f, c, box, shape, s, 1e-5, loss="sum", grads=False)["loss"]

    fd = (L(sig + h * d) - L(sig - h * d)) / (2 * h)
    an = np.sum(base["grad_sigma"] * d)
    assert abs(fd - an) <= 1e-5 * abs(an), (fd, an)
