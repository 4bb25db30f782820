"""Golden vectors at the benchmark configurations, from the reference's own CPU path.

Run once in a container that has the reference source checked out (read-only),
with ``$DELTAMIC_REF`` naming its root directory:

    DELTAMIC_REF=<reference checkout> python tests/golden/make_golden_configs.py

Cases (names start with ``cfg``; ``tests/test_gpu_configs.py`` and
``tests/test_oracle_configs.py`` read them):

* ``cfg1_icosphere_l3_64``: icosphere level 3 (642 vertices, 1,280 faces), radius
  0.3, vertices jittered by N(0, 0.01^2) (seed 2024), Faces_coeff 1,
  ``compute_box_size(verts, offset=0.2)``, 64^3, OTF = ``generate_gaussian_psf``
  with sigma 1e-3 I, narrow band 1e-5; forward, ``render_image_from_ftmesh``,
  ``normalize_tensor``, loss = sum(image), backward to Verts, Faces_coeff and
  sigma.  One call of ``Fourier3dMesh(device='cpu')`` (``MeshFTPy``,
  ``deltamic/render.py:36-109``) in float64 and in float32.
* ``cfg4_sh_l4_128``: icosphere level 4 (2,562 vertices, 5,120 faces) with a
  radial spherical-harmonic perturbation (l = 1..6, a_lm ~ N(0, (0.08/l)^2),
  seed 4), Faces_coeff ~ U(0.5, 1.5), 128^3, sigma 1e-3 I, band 1e-5, loss =
  mean((normalize(image) - target)^2) with ``oracle.smooth_target((128,)*3,
  seed=44)``.  The spectrum is evaluated in frequency chunks by masking the OTF
  argument (the chunks' spectra add up to the whole one), the loss and its
  gradient to the spectrum and to sigma are taken once on the summed spectrum,
  and each chunk is back-propagated with that spectrum gradient (the vertex and
  coefficient gradients add up over chunks).  Float64 and float32.

Stored: inputs, the band's voxel indices, the band spectrum, the loss, the
gradients (Verts, Faces_coeff, sigma), the float32 results with suffix ``_f32``,
image summaries (sum, min, max and 4,096 sampled voxels), and the oracle's
conditioning floor of the chain gradients (``oracle.chain_floor``) as
``floor_verts`` / ``floor_coeff`` / ``floor_sigma``.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402
from deltamic_b200.mesh import icosphere, jitter, random_sh_shape  # noqa: E402

REF = os.environ.get("DELTAMIC_REF", "")
CHUNK = 4096  # band frequencies per reference call (bounds its memory)


def _import_reference():
    if not REF or not os.path.isdir(os.path.join(REF, "deltamic")):
        raise SystemExit("set $DELTAMIC_REF to the root of a deltaMic checkout")
    sys.path.insert(0, REF)
    import deltamic.psf as psf  # noqa: E402
    import deltamic.render as render  # noqa: E402
    return psf, render


def make_cases():
    rng = np.random.default_rng(2024)
    v, f = icosphere(3, 0.3)
    v = jitter(v, 0.01, rng)
    cfg1 = dict(verts=v, faces=f, coeff=np.ones(len(f)), shape=(64, 64, 64),
                sigma=1e-3 * np.eye(3), thresh=1e-5, loss="sum", offset=0.2, chunk=None)
    v4, f4 = random_sh_shape(4, 0.3, 6, 0.08, seed=4)
    c4 = np.random.default_rng(40).uniform(0.5, 1.5, len(f4))
    cfg4 = dict(verts=v4, faces=f4, coeff=c4, shape=(128, 128, 128), sigma=1e-3 * np.eye(3),
                thresh=1e-5, loss="mse", offset=0.2, chunk=CHUNK, target_seed=44)
    return {"cfg1_icosphere_l3_64": cfg1, "cfg4_sh_l4_128": cfg4}


def run_reference(psf, render, case, dtype, target):
    shape = case["shape"]
    box = render.compute_box_size(case["verts"], offset=case["offset"])
    Verts = torch.tensor(case["verts"], dtype=dtype, requires_grad=True)
    Faces = torch.tensor(case["faces"], dtype=torch.long)
    coeff = torch.tensor(case["coeff"], dtype=dtype, requires_grad=True)
    sigma = torch.tensor(case["sigma"], dtype=dtype, requires_grad=True)
    mft = render.Fourier3dMesh(torch.tensor(box), shape, device="cpu", dtype=dtype,
                               narrowband_thresh=case["thresh"])
    otf = psf.generate_gaussian_psf(sigma, mft.xi0, mft.xi1, mft.xi2)
    band = (otf.detach().abs() > case["thresh"]).reshape(-1)
    idx = torch.nonzero(band).reshape(-1).numpy()
    tgt = None if target is None else torch.tensor(target, dtype=dtype)

    def chain(ft):
        img = render.render_image_from_ftmesh(ft, otf, shape)
        nimg = render.normalize_tensor(img)
        loss = nimg.sum() if case["loss"] == "sum" else torch.mean((nimg - tgt) ** 2)
        return img, loss

    if case["chunk"] is None:
        mft.OTF = otf.detach()
        ft = mft(Verts, Faces, coeff)
        ft.retain_grad()
        img, loss = chain(ft)
        loss.backward()
        grad_ft = ft.grad
    else:
        # chunks of the band: OTF argument zero outside the chunk
        chunks = [idx[k:k + case["chunk"]] for k in range(0, len(idx), case["chunk"])]
        flat = otf.detach().reshape(-1)

        def chunk_otf(c):
            o = torch.zeros_like(flat)
            o[torch.as_tensor(c)] = flat[torch.as_tensor(c)]
            return o.reshape(shape)

        with torch.no_grad():
            ft_sum = None
            for c in chunks:
                mft.OTF = chunk_otf(c)
                part = mft(Verts, Faces, coeff)
                ft_sum = part if ft_sum is None else ft_sum + part
        ft = ft_sum.detach().requires_grad_(True)
        img, loss = chain(ft)
        loss.backward()
        grad_ft = ft.grad
        for c in chunks:
            mft.OTF = chunk_otf(c)
            part = mft(Verts, Faces, coeff)
            part.backward(grad_ft)
    flat_img = img.detach().reshape(-1).numpy().astype(np.float64)
    samp = np.random.default_rng(7).choice(flat_img.size, 4096, replace=False)
    return dict(box=box, idx=idx,
                ft=ft.detach().reshape(-1)[band].numpy().astype(np.complex128),
                loss=float(loss.detach()),
                grad_verts=Verts.grad.numpy().astype(np.float64),
                grad_coeff=coeff.grad.numpy().astype(np.float64),
                grad_sigma=sigma.grad.numpy().astype(np.float64),
                image_sum=float(flat_img.sum()), image_min=float(flat_img.min()),
                image_max=float(flat_img.max()), image_sample_idx=samp.astype(np.int64),
                image_sample=flat_img[samp])


def main():
    psf, render = _import_reference()
    torch.set_num_threads(os.cpu_count() or 1)
    only = set(sys.argv[1:])
    for name, case in make_cases().items():
        if only and name not in only:
            continue
        target = (oracle.smooth_target(case["shape"], case["target_seed"])
                  if case["loss"] == "mse" else None)
        r64 = run_reference(psf, render, case, torch.float64, target)
        r32 = run_reference(psf, render, case, torch.float32, target)
        assert np.array_equal(r32["idx"], r64["idx"]), name
        out = dict(verts=case["verts"], faces=case["faces"], coeff=case["coeff"],
                   box_size=r64["box"], box_shape=np.array(case["shape"]),
                   sigma=case["sigma"], thresh=case["thresh"], loss_kind=case["loss"],
                   offset=case["offset"], idx=r64["idx"].astype(np.int32))
        if target is not None:
            out["target_seed"] = case["target_seed"]
        for k, v in r64.items():
            if k not in ("box", "idx"):
                out[k] = v
        for k in ("ft", "loss", "grad_verts", "grad_coeff", "grad_sigma", "image_sum",
                  "image_max"):
            v = r32[k]
            out[k + "_f32"] = v.astype(np.complex64) if k == "ft" else v
        fl = oracle.chain_floor(case["verts"], case["faces"], case["coeff"], r64["box"],
                                case["shape"], case["sigma"], case["thresh"], case["loss"],
                                target)
        out.update(floor_verts=fl["verts"], floor_coeff=fl["coeff"], floor_sigma=fl["sigma"])
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        print(f"{name}: nv={len(case['verts'])} nt={len(case['faces'])} "
              f"band={len(r64['idx'])} loss={r64['loss']:.6g} floor={fl} -> {path}", flush=True)


if __name__ == "__main__":
    main()
