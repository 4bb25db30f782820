"""Generate golden vectors for the autofluorescence (surface + enclosed volume)
transform by running the reference's own function.

Run once in a container that has the reference source checked out (read-only),
with ``$DELTAMIC_REF`` naming its root directory:

    DELTAMIC_REF=<reference checkout> python tests/golden/make_golden_volume.py

For every case it builds a small closed mesh and runs the reference's
``fourier_from_mesh_narrowband_autofluorescence`` (``deltamic/render.py:228-318``)
with torch autograd in float64, on the frequency axes of
``compute_spatial_frequency_grid`` (``render.py:321-340``) and the band
``OTF > thresh`` of ``generate_gaussian_psf`` (``deltamic/psf.py:15-20``).  The loss
is the fixed linear functional ``L = sum_band Re(conj(w) ft)`` with seeded complex
weights ``w`` (so ``w`` is the cotangent on the band).  Stored as
``volume_<case>.npz``: inputs, the band's voxel indices, ft on the band, and the
gradients with respect to Verts and regint.  On an odd grid the reference's
value at xi = 0 is 0/0 (NaN), so that case stores the forward only.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from deltamic_b200.mesh import icosphere, jitter, sh_perturb  # noqa: E402

REF = os.environ.get("DELTAMIC_REF", "")


def _import_reference():
    if not REF or not os.path.isdir(os.path.join(REF, "deltamic")):
        raise SystemExit("set $DELTAMIC_REF to the root of a deltaMic checkout")
    sys.path.insert(0, REF)
    import deltamic.psf as psf  # noqa: E402
    import deltamic.render as render  # noqa: E402
    return psf, render


def make_cases():
    rng = np.random.default_rng(2024)
    cases = {}
    v, f = icosphere(2, 0.3)
    cases["sphere_l2"] = dict(verts=jitter(v, 0.01, rng), faces=f, regint=0.5,
                              shape=(16, 16, 16), lengths=(1.0, 1.0, 1.0),
                              sigma=1e-3 * np.eye(3), thresh=1e-5, grads=True)
    v, f = icosphere(2, 0.3)
    v, _ = sh_perturb(v, 4, 0.08, rng, radius=0.3)
    cases["sh_aniso_shifted"] = dict(verts=v + np.array([0.21, -0.13, 0.07]), faces=f,
                                     regint=1.7, shape=(20, 18, 16), lengths=(1.2, 1.05, 0.9),
                                     sigma=np.diag([1e-3, 1.5e-3, 4e-3]), thresh=1e-5,
                                     grads=True)
    v, f = icosphere(1, 0.25)
    cases["odd_grid_forward"] = dict(verts=jitter(v, 0.01, rng), faces=f, regint=0.8,
                                     shape=(15, 15, 15), lengths=(1.0, 1.0, 1.0),
                                     sigma=2e-3 * np.eye(3), thresh=1e-5, grads=False)
    return cases


def run_reference(psf, render, case, rng):
    dt = torch.float64
    xi0, xi1, xi2 = render.compute_spatial_frequency_grid(case["shape"], case["lengths"],
                                                          dtype=dt)
    otf = psf.generate_gaussian_psf(torch.tensor(case["sigma"], dtype=dt), xi0, xi1, xi2)
    Verts = torch.tensor(case["verts"], dtype=dt, requires_grad=True)
    Faces = torch.tensor(case["faces"], dtype=torch.long)
    regint = torch.tensor(case["regint"], dtype=dt, requires_grad=True)
    ft = render.fourier_from_mesh_narrowband_autofluorescence(otf, case["thresh"], regint,
                                                              xi0, xi1, xi2, Verts, Faces)
    band = (otf > case["thresh"]).reshape(-1)
    idx = torch.nonzero(band).reshape(-1).numpy()
    ftb = ft.reshape(-1)[band]
    out = dict(idx=idx, ft=ftb.detach().numpy().astype(np.complex128))
    if case["grads"]:
        w = rng.normal(size=len(idx)) + 1j * rng.normal(size=len(idx))
        loss = torch.sum(torch.real(torch.conj(torch.tensor(w)) * ftb))
        loss.backward()
        out.update(w=w, grad_verts=Verts.grad.numpy().astype(np.float64),
                   grad_regint=float(regint.grad))
    return out


def main():
    psf, render = _import_reference()
    torch.set_num_threads(os.cpu_count() or 1)
    rng = np.random.default_rng(7)
    for name, case in make_cases().items():
        r = run_reference(psf, render, case, rng)
        out = dict(verts=case["verts"], faces=case["faces"], regint=case["regint"],
                   box_shape=np.array(case["shape"]), lengths=np.array(case["lengths"]),
                   sigma=case["sigma"], thresh=case["thresh"], **r)
        path = os.path.join(HERE, "volume_" + name + ".npz")
        np.savez_compressed(path, **out)
        print(f"{name}: nv={len(case['verts'])} nt={len(case['faces'])} band={len(r['idx'])} "
              f"nan={int(np.isnan(r['ft']).sum())} -> {path}")


if __name__ == "__main__":
    main()
