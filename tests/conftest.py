"""Shared test setup: the ``gpu`` marker, golden-fixture loading, tolerances."""
import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden_cases(prefix=""):
    """Fixture names under tests/golden: the small surface-transform cases (no
    prefix: every file not starting with ``volume_``, ``psf_`` or ``cfg``, the
    benchmark-configuration cases) or those starting with ``prefix``."""
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))
    if prefix:
        return [n for n in names if n.startswith(prefix)]
    return [n for n in names if not n.startswith(("volume_", "psf_", "cfg"))]


def load_golden(name):
    d = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
    return {k: d[k] for k in d.files}


def rel_l2(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


@pytest.fixture(params=golden_cases())
def golden(request):
    return request.param, load_golden(request.param)


@pytest.fixture(params=golden_cases("volume_"))
def golden_volume(request):
    return request.param, load_golden(request.param)


def band_xi(shape, lengths, idx):
    """xi[len(idx), 3] of the band's voxel indices on the centred grid of a box
    with the given lengths (render.py:321-340)."""
    axes = [(2 * np.arange(n) - (n - 1)) * np.pi / lengths[d] for d, n in enumerate(shape)]
    k = np.unravel_index(np.asarray(idx), tuple(shape))
    return np.stack([axes[d][k[d]] for d in range(3)], axis=1)
