"""Oracle: frequency grid, Gaussian OTF, narrow band, render, normalise, losses.

TEST INFRASTRUCTURE ONLY -- the checker for the CUDA path, never the product.

Follows, in numpy float64:

* ``Fourier3dMesh._compute_spatial_frequency_grid`` (``deltamic/render.py:153-172``):
  ``xi_d[k] = (2k - (n_d - 1)) * pi / (box[d,1] - box[d,0])``;
* ``generate_gaussian_psf`` (``deltamic/psf.py:15-20``): ``exp(-xi^T S xi / 2)``;
* the narrow band ``OTF > thresh`` of ``MeshFTCUDA.forward``
  (``deltamic/cuda_class.py:22-24``; the CPU path ``render.py:47`` takes ``abs``);
* ``render_image_from_ftmesh`` (``render.py:177-180``) and ``normalize_tensor``
  (``render.py:5-6``);
* the backward of that chain as torch autograd computes it: ``abs`` of a complex
  tensor (``g z/|z|``), the adjoint of ``ifftn`` (``fftn(g)/N``), the full-tensor
  ``min``/``max`` (gradient shared evenly by tied elements), and the Gaussian
  OTF's sigma gradient ``dL/dS_ij = sum_xi gOTF OTF (-xi_i xi_j / 2)``.
"""
from __future__ import annotations

import numpy as np

from .meshft import SEPS_F32, meshft_backward, meshft_forward


def compute_box_size(verts, offset=0.1):
    """render.py:9-18: cubic box around the vertices with ``offset`` extra extent."""
    verts = np.asarray(verts, np.float64)
    box = np.zeros((3, 2))
    extent = verts.max(axis=0) - verts.min(axis=0)
    box[:, 1] = verts.max(axis=0) + extent * offset / 2
    box[:, 0] = verts.min(axis=0) - extent * offset / 2
    box[:, 0] = box[:, 0].min(axis=0)
    box[:, 1] = box[:, 1].max(axis=0)
    return box


def frequency_axes(box_size, box_shape):
    box_size = np.asarray(box_size, np.float64)
    axes = []
    for d in range(3):
        n = int(box_shape[d])
        s = np.pi / (box_size[d, 1] - box_size[d, 0])
        axes.append((2.0 * np.arange(n) - (n - 1)) * s)
    return tuple(axes)


def gaussian_otf(sigma, xi0, xi1, xi2):
    s = np.asarray(sigma, np.float64)
    g0, g1, g2 = np.meshgrid(xi0, xi1, xi2, indexing="ij")
    q = (g0 * (s[0, 0] * g0 + s[0, 1] * g1 + s[0, 2] * g2)
         + g1 * (s[1, 0] * g0 + s[1, 1] * g1 + s[1, 2] * g2)
         + g2 * (s[2, 0] * g0 + s[2, 1] * g1 + s[2, 2] * g2))
    return np.exp(-q / 2.0)


def band_indices(otf, thresh, use_abs=False):
    """Flat C-order indices of the narrow band (boolean-mask order of torch)."""
    o = np.abs(otf) if use_abs else otf
    return np.flatnonzero(np.asarray(o).ravel() > thresh)


def xi_list_from_band(idx, axes):
    shape = tuple(len(a) for a in axes)
    k0, k1, k2 = np.unravel_index(idx, shape)
    return np.stack([axes[0][k0], axes[1][k1], axes[2][k2]], axis=1)


def render_from_band(ft_list, idx, otf):
    """|ifftn(ftmesh * OTF)| with ftmesh zero outside the band; returns (image, z)."""
    shape = otf.shape
    grid = np.zeros(shape, np.complex128)
    grid.ravel()[idx] = ft_list
    z = np.fft.ifftn(grid * otf)
    return np.abs(z), z


def normalize(t, c=0.0):
    return ((t - t.min()) / (t.max() - t.min()) + c) / (1.0 + c)


def image_loss(img, kind="sum", target=None, c=0.0):
    n = normalize(img, c)
    if kind == "sum":
        return float(n.sum())
    if kind == "mse":
        return float(np.mean((n - target) ** 2))
    raise ValueError(kind)


def image_loss_backward(img, kind="sum", target=None, c=0.0):
    """dL/dimg through ``normalize_tensor`` (min/max grads split among ties)."""
    mn, mx = img.min(), img.max()
    rng = mx - mn
    u = (img - mn) / rng
    n = (u + c) / (1.0 + c)
    if kind == "sum":
        gn = np.ones_like(img)
    elif kind == "mse":
        gn = 2.0 * (n - target) / img.size
    else:
        raise ValueError(kind)
    g = gn / (rng * (1.0 + c))
    d_mn = float(np.sum(gn * (-(1.0 - u)) / (rng * (1.0 + c))))
    d_mx = float(np.sum(gn * (-u) / (rng * (1.0 + c))))
    at_mn = img == mn
    at_mx = img == mx
    g = g + at_mn * (d_mn / at_mn.sum()) + at_mx * (d_mx / at_mx.sum())
    return g


def pipeline(verts, faces, coeff, box_size, box_shape, sigma, thresh,
             loss="sum", target=None, contrast=0.0, seps=SEPS_F32, threads=None,
             grads=True, ft_perturb=None):
    """Full oracle pass: OTF -> band -> meshFT -> render -> normalise -> loss.

    ``verts`` are in the box frame of the caller (unshifted); they are shifted by
    ``box_size[:,0]`` as ``Fourier3dMesh.forward`` does.  Returns a dict with the
    band indices, ``ft_list``, image, loss and (if ``grads``) the gradients with
    respect to verts, Faces_coeff and sigma.  ``ft_perturb(ft) -> ft`` replaces the
    spectrum before rendering (used to measure how strongly the gradients react
    to rounding-level changes of the spectrum).
    """
    box_size = np.asarray(box_size, np.float64)
    axes = frequency_axes(box_size, box_shape)
    otf = gaussian_otf(sigma, *axes)
    idx = band_indices(otf, thresh)
    xi = xi_list_from_band(idx, axes)
    v = np.asarray(verts, np.float64) - box_size[:, 0]
    ft = meshft_forward(v, faces, coeff, xi, seps=seps, threads=threads)
    if ft_perturb is not None:
        ft = ft_perturb(ft)
    img, z = render_from_band(ft, idx, otf)
    out = dict(idx=idx, xi=xi, ft=ft, otf=otf, image=img,
               loss=image_loss(img, loss, target, contrast))
    if not grads:
        return out
    gimg = image_loss_backward(img, loss, target, contrast)
    with np.errstate(invalid="ignore", divide="ignore"):
        gz = np.where(np.abs(z) > 0, gimg * z / np.abs(z), 0.0)
    gexp = np.fft.fftn(gz) / gz.size          # adjoint of ifftn
    gexp_band = gexp.ravel()[idx]
    otf_band = otf.ravel()[idx]
    g_ft = gexp_band * otf_band               # OTF is real
    g_otf = np.real(np.conj(gexp_band) * ft)  # zero outside the band
    gsig = np.empty((3, 3))
    for i in range(3):
        for j in range(3):
            gsig[i, j] = np.sum(g_otf * otf_band * (-0.5) * xi[:, i] * xi[:, j])
    gv, gc = meshft_backward(v, faces, coeff, xi, g_ft, ft, seps=seps, threads=threads)
    out.update(grad_verts=gv, grad_coeff=gc, grad_sigma=gsig, grad_ft=g_ft,
               grad_otf_band=g_otf)
    return out


def chain_floor(verts, faces, coeff, box_size, box_shape, sigma, thresh, loss="sum",
                target=None, rel=3e-7, trials=2, seed=0):
    """Conditioning floor of the render-chain gradients: the largest relative
    change of the (verts, coeff, sigma) gradients when the spectrum is perturbed by
    complex noise of relative size ``rel`` (float32 rounding level)."""
    base = pipeline(verts, faces, coeff, box_size, box_shape, sigma, thresh, loss, target)
    rng = np.random.default_rng(seed)
    worst = np.zeros(3)

    def rl(a, b):
        return np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)

    for _ in range(trials):
        def pert(ft):
            n = rng.normal(size=ft.shape) + 1j * rng.normal(size=ft.shape)
            return ft + n * np.abs(ft) * rel
        o = pipeline(verts, faces, coeff, box_size, box_shape, sigma, thresh, loss, target,
                     ft_perturb=pert)
        worst = np.maximum(worst, [rl(o["grad_verts"], base["grad_verts"]),
                                   rl(o["grad_coeff"], base["grad_coeff"]),
                                   rl(o["grad_sigma"], base["grad_sigma"])])
    return dict(verts=float(worst[0]), coeff=float(worst[1]), sigma=float(worst[2]))


def smooth_target(box_shape, seed, width=0.15, noise=0.05):
    """Deterministic target image for image-L2 losses: a Gaussian blob at the box
    centre (width relative to the box) plus N(0, noise^2) voxel noise from
    numpy's PCG64 with ``seed``; float64, the same array on every machine."""
    u = [np.arange(n, dtype=np.float64) / max(n - 1, 1) - 0.5 for n in box_shape]
    r2 = u[0][:, None, None] ** 2 + u[1][None, :, None] ** 2 + u[2][None, None, :] ** 2
    t = np.exp(-r2 / (2.0 * width * width))
    rng = np.random.default_rng(seed)
    return t + noise * rng.standard_normal(tuple(box_shape))
