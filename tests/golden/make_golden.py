"""Generate golden vectors by running the reference deltaMic CPU path.

Run once in a container that has the reference source checked out (read-only),
with ``$DELTAMIC_REF`` naming its root directory:

    DELTAMIC_REF=<reference checkout> python tests/golden/make_golden.py

For every case it builds a small mesh, then runs the reference's own
``Fourier3dMesh(device='cpu')`` (i.e. ``MeshFTPy``, ``deltamic/render.py:36-109``),
``generate_gaussian_psf`` (``deltamic/psf.py:15-20``), ``render_image_from_ftmesh``
and ``normalize_tensor`` with torch autograd, in float64 and in float32, and
stores inputs and outputs (narrow-band ft list, image, loss, gradients with
respect to Verts, Faces_coeff and sigma) as ``<case>.npz`` next to this script.
The GPU tests never import the reference; they only read these files.
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


def cube_mesh(lo, hi):
    """Axis-aligned box surface (12 triangles): edges parallel to the axes force
    exact zero phase differences (branches R1..R4) whenever a grid frequency
    component is 0 (odd box_shape)."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], np.float64)
    f = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                  [1, 2, 6], [1, 6, 5], [2, 3, 7], [2, 7, 6], [3, 0, 4], [3, 4, 7]],
                 np.int64)
    return v, f


def make_cases():
    cases = {}
    rng = np.random.default_rng(1234)

    v, f = icosphere(1, 0.3)
    v = jitter(v, 0.01, rng)
    cases["sphere_l1_sum"] = dict(verts=v, faces=f, coeff=np.ones(len(f)),
                                  shape=(16, 16, 16), sigma=1e-3 * np.eye(3),
                                  thresh=1e-5, loss="sum", offset=0.2)

    v, f = icosphere(2, 0.3)
    v, _ = sh_perturb(v, 4, 0.08, rng, radius=0.3)
    vt, _ = sh_perturb(icosphere(2, 0.3)[0], 4, 0.08, rng, radius=0.3)
    cases["sh_l2_aniso_mse"] = dict(verts=v, faces=f, coeff=rng.uniform(0.5, 1.5, len(f)),
                                    shape=(20, 18, 16),
                                    sigma=np.diag([1e-3, 1e-3, 4e-3]),
                                    thresh=1e-5, loss="mse", offset=0.2, target_verts=vt)

    v, f = icosphere(2, 0.25)
    v = jitter(v, 0.01, rng)
    cases["odd_grid_fullsigma"] = dict(
        verts=v, faces=f, coeff=rng.uniform(0.5, 1.5, len(f)), shape=(21, 21, 21),
        sigma=np.array([[1.0e-3, 2.0e-4, 0.0], [2.0e-4, 1.5e-3, 1.0e-4],
                        [0.0, 1.0e-4, 2.0e-3]]),
        thresh=1e-4, loss="sum", offset=0.2)

    v, f = cube_mesh((-0.2, -0.15, -0.1), (0.2, 0.15, 0.25))
    # random per-face coefficients break the mirror symmetry of the box, so the
    # rendered image has a unique maximum (tied extrema make the normalize_tensor
    # gradient depend on last-bit rounding)
    cases["cube_degenerate"] = dict(verts=v, faces=f, coeff=rng.uniform(0.5, 1.5, len(f)),
                                    shape=(15, 15, 15), sigma=2e-3 * np.eye(3),
                                    thresh=1e-5, loss="sum", offset=0.4)
    return cases


def run_reference(psf, render, case, dtype, target=None):
    verts = case["verts"]
    box = render.compute_box_size(verts, offset=case["offset"])
    Verts = torch.tensor(verts, dtype=dtype, requires_grad=True)
    Faces = torch.tensor(case["faces"], dtype=torch.long)
    coeff = torch.tensor(case["coeff"], dtype=dtype, requires_grad=True)
    sigma = torch.tensor(case["sigma"], dtype=dtype, requires_grad=True)
    mft = render.Fourier3dMesh(torch.tensor(box), case["shape"], device="cpu", dtype=dtype,
                               narrowband_thresh=case["thresh"])
    otf = psf.generate_gaussian_psf(sigma, mft.xi0, mft.xi1, mft.xi2)
    mft.OTF = otf.detach()
    ft = mft(Verts, Faces, coeff)
    ft.retain_grad()
    img = render.render_image_from_ftmesh(ft, otf, case["shape"])
    img.retain_grad()
    nimg = render.normalize_tensor(img)
    if case["loss"] == "sum":
        loss = nimg.sum()
    else:
        loss = torch.mean((nimg - torch.tensor(target, dtype=dtype)) ** 2)
    loss.backward()
    band = (otf.detach().abs() > case["thresh"]).reshape(-1)
    idx = torch.nonzero(band).reshape(-1).numpy()
    return dict(box=box, idx=idx,
                ft=ft.detach().reshape(-1)[band].numpy().astype(np.complex128),
                image=img.detach().numpy().astype(np.float64),
                loss=float(loss.detach()),
                grad_verts=Verts.grad.numpy().astype(np.float64),
                grad_coeff=coeff.grad.numpy().astype(np.float64),
                grad_sigma=sigma.grad.numpy().astype(np.float64),
                grad_ft=ft.grad.reshape(-1)[band].numpy().astype(np.complex128))


def main():
    psf, render = _import_reference()
    torch.set_num_threads(os.cpu_count() or 1)
    for name, case in make_cases().items():
        target = None
        if case["loss"] == "mse":
            # target image: the reference render of a different shape, normalised
            tc = dict(case, verts=case["target_verts"])
            box = render.compute_box_size(case["verts"], offset=case["offset"])
            mft = render.Fourier3dMesh(torch.tensor(box), case["shape"], device="cpu",
                                       dtype=torch.float64, narrowband_thresh=case["thresh"])
            otf = psf.generate_gaussian_psf(torch.tensor(case["sigma"]), mft.xi0, mft.xi1, mft.xi2)
            mft.OTF = otf
            ftt = mft(torch.tensor(tc["verts"]), torch.tensor(case["faces"]),
                      torch.tensor(case["coeff"]))
            target = render.normalize_tensor(
                render.render_image_from_ftmesh(ftt, otf, case["shape"])).numpy()
        r64 = run_reference(psf, render, case, torch.float64, target)
        r32 = run_reference(psf, render, case, torch.float32, target)
        out = dict(verts=case["verts"], faces=case["faces"], coeff=case["coeff"],
                   box_size=r64["box"], box_shape=np.array(case["shape"]),
                   sigma=case["sigma"], thresh=case["thresh"], loss_kind=case["loss"],
                   offset=case["offset"])
        if target is not None:
            out["target"] = target
        for k, v in r64.items():
            if k != "box":
                out[k] = v
        for k, v in r32.items():
            if k not in ("box", "idx"):
                out[k + "_f32"] = v
        assert np.array_equal(r32["idx"], r64["idx"]), name
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        print(f"{name}: nv={len(case['verts'])} nt={len(case['faces'])} "
              f"band={len(r64['idx'])} loss={r64['loss']:.6g} -> {path}")


if __name__ == "__main__":
    main()
