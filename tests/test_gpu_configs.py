"""Parity at the benchmark configurations, on the GPU, against the float64 oracle and
the reference's own outputs (golden vectors from tests/golden/make_golden_configs.py).

* cfg1 (level-3 icosphere, 64^3, sum of the normalised image): the drop-in chain
  Fourier3dMesh -> render_image_from_ftmesh -> normalize_tensor -> loss ->
  backward against the reference's float64 run (float32 kernels, and the float64
  module).
* cfg2 (level-5 SH mesh, 20,480 faces, 200^3, sigma diag(1e-3, 1e-3, 4e-3)): the
  full-band forward and the full adjoint (vertex and coefficient gradients) with a
  cotangent supported on 384 band frequencies, against the oracle on those
  frequencies (the adjoint is linear in the cotangent, so the oracle needs only
  them); the whole spectrum through size-independent checks.
* cfg3 (64 cells, levels 2-5, 64/96/128^3, per-cell sigma and coefficients): every
  cell's spectrum and adjoint from the batched launches against the oracle on a
  48-frequency sample of that cell.
* cfg4 (level-4 SH mesh, 128^3, random coefficients, image L2): gradients to the
  vertices, Faces_coeff and the sigma diagonal against the reference's float64
  gradient and against float64 central finite differences (200 directional probes,
  step 1e-6 relative; loss evaluated by the float64 module with the band fixed),
  and the adjoint's device memory against a stored phase table.

Every test prints its rel-L2 against float64 and, where the golden holds one, the
reference float32's own distance from float64."""
import ctypes
import os

import numpy as np
import pytest
import torch

import oracle
from conftest import GOLDEN_DIR, load_golden, rel_l2
from deltamic_b200 import _native as N
from deltamic_b200 import ops
from deltamic_b200.mesh import icosphere, random_sh_shape

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL_FT, TOL_GV, TOL_GC = 1e-5, 1e-4, 1e-5
TOL_CHAIN_V, TOL_CHAIN = 2e-4, 1e-4


def _t(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def _have(name):
    return os.path.exists(os.path.join(GOLDEN_DIR, name + ".npz"))


def _chain(d, dtype, target=None):
    """The drop-in chain on golden d's inputs; returns (ft, img, loss, V, C, S, mft)."""
    import deltamic_b200 as dm
    shape = tuple(int(s) for s in d["box_shape"])
    V = _t(d["verts"], dtype).requires_grad_(True)
    C = _t(d["coeff"], dtype).requires_grad_(True)
    S = _t(d["sigma"], dtype).requires_grad_(True)
    mft = dm.Fourier3dMesh(torch.tensor(d["box_size"]), shape, device=DEV, dtype=dtype,
                           narrowband_thresh=float(d["thresh"]))
    otf = dm.generate_gaussian_psf(S, mft.xi0, mft.xi1, mft.xi2)
    mft.OTF = otf.detach()
    ft = mft(V, _t(d["faces"], torch.int64), C)
    img = dm.render_image_from_ftmesh(ft, otf, shape)
    nimg = dm.normalize_tensor(img)
    if str(d["loss_kind"]) == "sum":
        loss = nimg.sum()
    else:
        loss = torch.mean((nimg - _t(target, dtype)) ** 2)
    loss.backward()
    return ft, img, loss, V, C, S, mft


@pytest.mark.skipif(not _have("cfg1_icosphere_l3_64"), reason="golden not generated")
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_cfg1_chain_against_reference(dtype):
    d = load_golden("cfg1_icosphere_l3_64")
    ft, img, loss, V, C, S, mft = _chain(d, dtype)
    band = mft.band().cpu().numpy()
    common, ia, ib = np.intersect1d(band, d["idx"], return_indices=True)
    assert len(common) >= 0.999 * len(d["idx"])
    e_ft = rel_l2(ft.detach().reshape(-1).cpu().numpy()[common], d["ft"][ib])
    im = img.detach().reshape(-1).cpu().numpy()
    e_img = rel_l2(im[d["image_sample_idx"]], d["image_sample"])
    ev = rel_l2(V.grad.cpu().numpy(), d["grad_verts"])
    ec = rel_l2(C.grad.cpu().numpy(), d["grad_coeff"])
    es = rel_l2(S.grad.cpu().numpy(), d["grad_sigma"])
    print(f"cfg1 {dtype}: vs reference float64 ft {e_ft:.2e} image {e_img:.2e} verts {ev:.2e} "
          f"coeff {ec:.2e} sigma {es:.2e}; reference float32 vs float64: ft "
          f"{rel_l2(d['ft_f32'], d['ft']):.2e} verts "
          f"{rel_l2(d['grad_verts_f32'], d['grad_verts']):.2e} coeff "
          f"{rel_l2(d['grad_coeff_f32'], d['grad_coeff']):.2e} sigma "
          f"{rel_l2(d['grad_sigma_f32'], d['grad_sigma']):.2e}")
    rl = abs(float(loss.detach()) - float(d["loss"])) / abs(float(d["loss"]))
    if dtype == torch.float64:
        # float64 kernels: the reference's CPU float64 arithmetic (same Seps)
        assert e_ft < 1e-9 and e_img < 1e-9 and rl < 1e-9
        assert ev < 1e-6 and ec < 1e-8 and es < 1e-8
    else:
        assert e_ft < TOL_FT and e_img < TOL_FT and rl < 1e-4
        assert ev < max(TOL_CHAIN_V, 2 * float(d["floor_verts"]))
        assert ec < max(TOL_CHAIN, 2 * float(d["floor_coeff"]))
        assert es < max(TOL_CHAIN, 2 * float(d["floor_sigma"]))


def test_cfg2_full_size_adjoint_against_oracle():
    v, f = random_sh_shape(5, 0.3, 6, 0.08, seed=1234)
    c = np.random.default_rng(12).uniform(0.5, 1.5, len(f))
    box = oracle.compute_box_size(v, 0.2)
    shape = (200, 200, 200)
    grid = ops.FreqGrid(box, shape)
    xi = grid.axes(torch.float32, DEV)
    otf = ops.gaussian_otf(_t(np.diag([1e-3, 1e-3, 4e-3])), *xi)
    band = ops.narrowband(otf, 1e-5)
    assert ops.band_is_hermitian(band)
    nb = band.numel()
    V, F, C = _t(v), _t(f, torch.int64), _t(c)
    ft = ops.meshft_list(V, F, C, grid, band)
    rng = np.random.default_rng(21)
    sub = np.sort(rng.choice(nb, 384, replace=False))
    g = np.zeros(nb, np.complex64)
    g[sub] = (rng.normal(size=len(sub)) + 1j * rng.normal(size=len(sub))).astype(np.complex64)
    gv, gc, _ = ops.meshft_backward_list(V, F, C, grid, band, ft, grad_list=_t(g, torch.complex64))
    idx = band.cpu().numpy().astype(np.int64)
    xil = oracle.xi_list_from_band(idx[sub], oracle.frequency_axes(box, shape))
    vs = v - box[:, 0]
    ft64 = oracle.meshft_forward(vs, f, c, xil)
    rv, rc = oracle.meshft_backward(vs, f, c, xil, g[sub], ft64)
    ftn = ft.cpu().numpy()
    e_ft, e_gv, e_gc = rel_l2(ftn[sub], ft64), rel_l2(gv.cpu().numpy(), rv), rel_l2(
        gc.cpu().numpy(), rc)
    print(f"cfg2 (200^3, 20,480 faces, band {nb}): ft {e_ft:.2e} verts {e_gv:.2e} "
          f"coeff {e_gc:.2e} against float64 on {len(sub)} frequencies")
    assert e_ft < TOL_FT and e_gv < TOL_GV and e_gc < TOL_GC
    # whole spectrum: mirror symmetry ft(-xi) = conj(ft(xi)) and the coefficient
    # scale invariance sum_k c_k dL/dc_k = 0 (ft does not change when all c scale)
    assert np.array_equal(ftn[::-1], np.conj(ftn))
    s = float(np.dot(c, gc.cpu().numpy().astype(np.float64)))
    assert abs(s) < 1e-4 * np.abs(c * gc.cpu().numpy()).sum()


def test_cfg3_every_cell_against_oracle():
    from deltamic_b200.batch import BatchRenderer
    rng = np.random.default_rng(4242)
    cells = []
    for i in range(64):
        level = int(rng.integers(2, 6))
        n = int(rng.choice([64, 96, 128]))
        v, f = random_sh_shape(level, 0.3, 6, 0.08, seed=int(rng.integers(1 << 30)))
        cells.append(dict(v=v, f=f, c=rng.uniform(0.5, 1.5, len(f)),
                          box=oracle.compute_box_size(v, 0.2), shape=(n, n, n),
                          sigma=np.diag(rng.uniform(5e-4, 4e-3, 3))))
    br = BatchRenderer([x["box"] for x in cells], [x["shape"] for x in cells], 1e-5, DEV)
    br.set_sigmas([x["sigma"] for x in cells])
    br.set_meshes([x["v"] for x in cells], [x["f"] for x in cells])
    V = _t(np.concatenate([x["v"] for x in cells]))
    C = _t(np.concatenate([x["c"] for x in cells]))
    ft = br.forward_spectrum(V, C)
    offs = np.concatenate([[0], np.cumsum(br.band_sizes)])
    g = np.zeros(br.band.numel(), np.complex64)
    samples = []
    for i in range(64):
        s = np.sort(rng.choice(br.band_sizes[i], min(48, br.band_sizes[i]), replace=False))
        g[offs[i] + s] = (rng.normal(size=len(s)) + 1j * rng.normal(size=len(s)))
        samples.append(s)
    lib = N.lib()
    gv = torch.empty_like(V)
    gc = torch.empty_like(C)
    w = br._ws["bwd_workspace"]
    N.check(lib.dm_batched_meshft_backward(
        ctypes.byref(br.batch), N.ptr(V), N.ptr(br.faces), N.ptr(C), N.ptr(br.band),
        N.ptr(_t(g, torch.complex64)), None, None, 1.0, N.ptr(ft), N.ptr(br._topo), N.ptr(gv),
        N.ptr(gc), None, N.ptr(w), w.numel(), N.stream_ptr(DEV)), "dm_batched_meshft_backward")
    ftn, gvn, gcn = ft.cpu().numpy(), gv.cpu().numpy(), gc.cpu().numpy()
    band = br.band.cpu().numpy().astype(np.int64)
    vo = np.concatenate([[0], np.cumsum([len(x["v"]) for x in cells])])
    fo = np.concatenate([[0], np.cumsum([len(x["f"]) for x in cells])])
    worst = np.zeros(3)
    for i, x in enumerate(cells):
        s = samples[i]
        idx = band[offs[i]:offs[i + 1]][s]
        xil = oracle.xi_list_from_band(idx, oracle.frequency_axes(x["box"], x["shape"]))
        vs = x["v"] - x["box"][:, 0]
        ft64 = oracle.meshft_forward(vs, x["f"], x["c"], xil)
        rv, rc = oracle.meshft_backward(vs, x["f"], x["c"], xil, g[offs[i] + s], ft64)
        e = [rel_l2(ftn[offs[i] + s], ft64), rel_l2(gvn[vo[i]:vo[i + 1]], rv),
             rel_l2(gcn[fo[i]:fo[i + 1]], rc)]
        worst = np.maximum(worst, e)
        assert e[0] < TOL_FT and e[1] < TOL_GV and e[2] < TOL_GC, (i, e)
    print(f"cfg3 64 cells: worst cell ft {worst[0]:.2e} verts {worst[1]:.2e} "
          f"coeff {worst[2]:.2e} against float64 (48 frequencies per cell)")


def _cfg4_loss64(d, target, band_otf, dv=None, dc=None, ds=None):
    """Float64 loss of the cfg4 chain at perturbed parameters (band fixed to the
    base OTF's, as the gradient treats it)."""
    import deltamic_b200 as dm
    shape = tuple(int(s) for s in d["box_shape"])
    V = _t(d["verts"], torch.float64) + (0 if dv is None else dv)
    C = _t(d["coeff"], torch.float64) + (0 if dc is None else dc)
    S = _t(d["sigma"], torch.float64) + (0 if ds is None else torch.diag(ds))
    mft = dm.Fourier3dMesh(torch.tensor(d["box_size"]), shape, device=DEV, dtype=torch.float64,
                           narrowband_thresh=float(d["thresh"]))
    mft.OTF = band_otf
    with torch.no_grad():
        otf = dm.generate_gaussian_psf(S, mft.xi0, mft.xi1, mft.xi2)
        ft = mft(V, _t(d["faces"], torch.int64), C)
        img = dm.render_image_from_ftmesh(ft, otf, shape)
        return float(torch.mean((dm.normalize_tensor(img) - target) ** 2))


@pytest.mark.skipif(not _have("cfg4_sh_l4_128"), reason="golden not generated")
def test_cfg4_adjoint_against_reference_and_fp64_finite_differences():
    d = load_golden("cfg4_sh_l4_128")
    shape = tuple(int(s) for s in d["box_shape"])
    target = oracle.smooth_target(shape, int(d["target_seed"]))
    # float32 product path, with the adjoint's peak memory
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats()
    base = torch.cuda.memory_allocated()
    ft, img, loss, V, C, S, mft = _chain(d, torch.float32, target)
    torch.cuda.synchronize()
    peak = torch.cuda.max_memory_allocated() - base
    g32 = [V.grad.double(), C.grad.double(), torch.diagonal(S.grad).double()]
    # float64 product path
    _, _, loss64, V6, C6, S6, mft64 = _chain(d, torch.float64, target)
    g64 = [V6.grad, C6.grad, torch.diagonal(S6.grad)]
    ref = [d["grad_verts"], d["grad_coeff"], np.diag(d["grad_sigma"])]
    ref32 = [d["grad_verts_f32"], d["grad_coeff_f32"], np.diag(d["grad_sigma_f32"])]
    names = ("verts", "coeff", "sigma_diag")
    for n, a, b, r, r32 in zip(names, g32, g64, ref, ref32):
        print(f"cfg4 {n}: float32 path vs reference float64 {rel_l2(a.cpu().numpy(), r):.2e}, "
              f"float64 path {rel_l2(b.cpu().numpy(), r):.2e}; reference float32 "
              f"{rel_l2(r32, r):.2e}")
    fl = [float(d["floor_verts"]), float(d["floor_coeff"]), float(d["floor_sigma"])]
    assert rel_l2(g32[0].cpu().numpy(), ref[0]) < max(TOL_CHAIN_V, 2 * fl[0])
    assert rel_l2(g32[1].cpu().numpy(), ref[1]) < max(TOL_CHAIN, 2 * fl[1])
    assert rel_l2(g32[2].cpu().numpy(), ref[2]) < max(TOL_CHAIN, 2 * fl[2])
    for b, r in zip(g64, ref):
        assert rel_l2(b.cpu().numpy(), r) < 1e-6
    # 200 directional probes: 80 vertex, 60 coefficient, 60 sigma-diagonal directions
    tgt = _t(target, torch.float64)
    band_otf = mft64.OTF
    rng = np.random.default_rng(400)
    x0 = [_t(d["verts"], torch.float64), _t(d["coeff"], torch.float64),
          _t(np.diag(d["sigma"]), torch.float64)]
    fd, an32, an64 = [], [], []
    for grp, count in ((0, 80), (1, 60), (2, 60)):
        for _ in range(count):
            u = _t(rng.normal(size=x0[grp].shape), torch.float64)
            u = u / torch.linalg.norm(u)
            h = 1e-6 * float(torch.linalg.norm(x0[grp]))
            key = ("dv", "dc", "ds")[grp]
            lp = _cfg4_loss64(d, tgt, band_otf, **{key: h * u})
            lm = _cfg4_loss64(d, tgt, band_otf, **{key: -h * u})
            fd.append((lp - lm) / (2 * h))
            an32.append(float((g32[grp] * u).sum()))
            an64.append(float((g64[grp] * u).sum()))
    fd, an32, an64 = map(np.asarray, (fd, an32, an64))
    groups = [slice(0, 80), slice(80, 140), slice(140, 200)]
    for n, sl, f in zip(names, groups, fl):
        e32 = rel_l2(an32[sl], fd[sl])
        e64 = rel_l2(an64[sl], fd[sl])
        print(f"cfg4 FD ({n}, {sl.stop - sl.start} probes, step 1e-6 relative): "
              f"float32 adjoint {e32:.2e}, float64 adjoint {e64:.2e}")
        assert e64 < 1e-5
        assert e32 < max(2e-3, 3 * f)
    # memory: the recompute adjoint against a stored per-pair phase table
    n_xi, nt = len(d["idx"]), len(d["faces"])
    table = 3 * n_xi * nt * 8  # three complex64 exponentials per (frequency, face)
    lib = N.lib()
    ws = int(lib.dm_meshft_backward_workspace_size(len(d["verts"]), nt, n_xi))
    print(f"cfg4 memory: adjoint workspace {ws / 2**20:.1f} MiB, peak device memory of the "
          f"whole float32 forward+backward chain {peak / 2**20:.1f} MiB; a stored phase "
          f"table would take {table / 2**30:.2f} GiB ({table / max(ws, 1):.0f}x the workspace)")
    assert ws < table / 100
