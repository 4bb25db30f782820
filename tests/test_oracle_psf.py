"""Oracle of the spatial PSF models (deltamic/psf.py) against golden vectors made
by the reference modules themselves (tests/golden/make_golden_psf.py)."""
import numpy as np
import pytest

import oracle.psf as op
from conftest import load_golden, rel_l2
from deltamic_b200 import noll2degrees


def _axes(g):
    sh, sz = tuple(int(v) for v in g["box_shape"]), g["box_size"]
    return [np.linspace(-sz[d] / 2, sz[d] / 2, sh[d], dtype=np.float32).astype(np.float64)
            for d in range(3)]


def test_noll_degrees_and_zernike_match_reference():
    g = load_golden("psf_zernike")
    n, m = noll2degrees(np.arange(1, 67))
    assert np.array_equal(n, g["n"]) and np.array_equal(m, g["m"])
    Z = np.array([op.zernike_explicit(g["r"], g["theta"], a, b) for a, b in zip(n, m)])
    assert np.max(np.abs(Z - g["z"])) < 1e-11


def test_aniso_gaussian_matches_reference():
    g = load_golden("psf_aniso")
    P = op.aniso_gaussian_psf(*_axes(g), g["sigma"], float(g["sigma_z"]), float(g["eps"]))
    assert rel_l2(P, g["psf"]) < 1e-6


@pytest.mark.parametrize("case", ["psf_gl_default", "psf_gl_custom"])
def test_gibson_lanni_radial_decomposition_matches_reference(case):
    """One Fourier-Bessel amplitude per distinct pixel radius, scattered: the
    reference's per-pixel PSF to the conditioning of its least-squares fit."""
    g = load_golden(case)
    kw = {str(k): float(v) for k, v in zip(g["kwargs_keys"], g["kwargs_vals"])}
    P = op.gibson_lanni_radial(tuple(int(v) for v in g["box_shape"]), **kw)
    assert rel_l2(P, g["psf"]) < 1e-9


def test_hanser_matches_reference():
    g = load_golden("psf_hanser")
    f32 = lambda a: np.asarray(a, np.float32).astype(np.float64)
    P = op.hanser_psf(tuple(int(v) for v in g["box_shape"]), f32(g["pcoefs"]), f32(g["mcoefs"]),
                      res_axial=float(g["res_axial"]))
    assert rel_l2(P, g["psf"]) < 1e-5
