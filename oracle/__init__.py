"""CPU oracle for the deltaMic render-and-fit hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, in numpy float64, the arithmetic of the reference
implementation (deltamic ``render.py``, ``psf.py`` and the adjoint of
``cpp/fourier3d_cuda_kernel.cu``).  It is the checker for the CUDA product path:
only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it.  Nothing in
``deltamic_b200`` imports it, and the product path never falls back to it.

Parity pin: ``tests/golden/make_golden.py`` ran the reference's own CPU path
(``deltamic.render.MeshFTPy`` with torch autograd, float64) on small meshes and
stored inputs/outputs under ``tests/golden/``; ``tests/test_oracle_golden.py``
checks this oracle against those vectors.
"""
from .meshft import (SEPS_F32, SEPS_F64, face_areas, pair_F, pair_F_and_grads,
                     meshft_forward, meshft_backward)
from .render import (frequency_axes, gaussian_otf, band_indices, xi_list_from_band,
                     render_from_band, normalize, image_loss, image_loss_backward,
                     pipeline, chain_floor, compute_box_size, smooth_target)
from . import fit

__all__ = [
    "SEPS_F32", "SEPS_F64", "face_areas", "pair_F", "pair_F_and_grads",
    "meshft_forward", "meshft_backward", "frequency_axes", "gaussian_otf",
    "band_indices", "xi_list_from_band", "render_from_band", "normalize",
    "image_loss", "image_loss_backward", "pipeline", "chain_floor", "compute_box_size", "fit",
    "smooth_target",
]
