"""CUDA meshFT forward / adjoint against the float64 oracle and the reference's
golden vectors.  Tolerances (rel-L2, float32 kernels vs float64):
  ft_list 1e-5, vertex gradient 1e-4, Faces_coeff gradient 1e-5 for the meshFT
  adjoint with a given cotangent; through the whole float32 render chain (FFT,
  |.|, normalize, loss) 2e-4 (vertices) and 1e-4 (Faces_coeff, sigma), or twice
  the chain's conditioning floor where that is larger (oracle.chain_floor)."""
import numpy as np
import pytest
import torch

import oracle
from conftest import load_golden, rel_l2
from deltamic_b200 import ops
from deltamic_b200.mesh import icosphere, jitter, random_sh_shape

pytestmark = pytest.mark.gpu

TOL_FT = 1e-5
TOL_GV = 1e-4
TOL_GC = 1e-5
TOL_CHAIN_V = 2e-4
TOL_CHAIN = 1e-4

DEV = "cuda:0"


def _t(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def _setup(v, f, c, box, shape, sigma, thresh):
    grid = ops.FreqGrid(box, shape)
    xi = grid.axes(torch.float32, DEV)
    otf = ops.gaussian_otf(_t(sigma), *xi)
    band = ops.narrowband(otf, thresh)
    return grid, xi, otf, band


def _oracle_xi(grid, band):
    axes = oracle.frequency_axes(grid.box_size, grid.shape)
    return oracle.xi_list_from_band(band.cpu().numpy().astype(np.int64), axes)


def _case(level=2, shape=(24, 24, 24), seed=0, sigma=None, thresh=1e-5):
    v, f = random_sh_shape(level, 0.3, 4, 0.08, seed)
    rng = np.random.default_rng(seed + 100)
    c = rng.uniform(0.5, 1.5, len(f))
    box = oracle.compute_box_size(v, 0.2)
    sigma = np.diag([1e-3, 1e-3, 4e-3]) if sigma is None else sigma
    return v, f, c, box, shape, sigma, thresh


@pytest.mark.parametrize("level,shape", [(1, (16, 16, 16)), (2, (24, 20, 18)), (3, (33, 33, 33))])
def test_forward_matches_oracle(level, shape):
    v, f, c, box, shape, sigma, thresh = _case(level, shape)
    grid, xi, otf, band = _setup(v, f, c, box, shape, sigma, thresh)
    ft = ops.meshft_list(_t(v), _t(f, torch.int64), _t(c), grid, band)
    xil = _oracle_xi(grid, band)
    ref = oracle.meshft_forward(v - box[:, 0], f, c, xil)
    assert rel_l2(ft.cpu().numpy(), ref) < TOL_FT


@pytest.mark.parametrize("level,shape", [(1, (16, 16, 16)), (2, (24, 20, 18)), (3, (25, 25, 25))])
def test_backward_matches_oracle(level, shape):
    v, f, c, box, shape, sigma, thresh = _case(level, shape, seed=1)
    grid, xi, otf, band = _setup(v, f, c, box, shape, sigma, thresh)
    V, F, C = _t(v), _t(f, torch.int64), _t(c)
    ft = ops.meshft_list(V, F, C, grid, band)
    rng = np.random.default_rng(7)
    g = (rng.normal(size=band.numel()) + 1j * rng.normal(size=band.numel()))
    g = g * np.exp(-0.5 * np.linalg.norm(_oracle_xi(grid, band), axis=1) ** 2 * 1e-4)
    gv, gc, _ = ops.meshft_backward_list(V, F, C, grid, band, ft,
                                         grad_list=_t(g, torch.complex64))
    xil = _oracle_xi(grid, band)
    ft64 = oracle.meshft_forward(v - box[:, 0], f, c, xil)
    rv, rc = oracle.meshft_backward(v - box[:, 0], f, c, xil, g.astype(np.complex64), ft64)
    assert rel_l2(gv.cpu().numpy(), rv) < TOL_GV
    assert rel_l2(gc.cpu().numpy(), rc) < TOL_GC


def test_drop_in_chain_matches_reference_golden(golden):
    """Fourier3dMesh -> render_image_from_ftmesh -> normalize_tensor -> loss ->
    backward, against the reference's float64 autograd (golden vectors)."""
    import deltamic_b200 as dm
    name, d = golden
    shape = tuple(int(s) for s in d["box_shape"])
    V = _t(d["verts"]).requires_grad_(True)
    F = _t(d["faces"], torch.int64)
    C = _t(d["coeff"]).requires_grad_(True)
    S = _t(d["sigma"]).requires_grad_(True)
    mft = dm.Fourier3dMesh(torch.tensor(d["box_size"]), shape, device=DEV,
                           narrowband_thresh=float(d["thresh"]))
    otf = dm.generate_gaussian_psf(S, mft.xi0, mft.xi1, mft.xi2)
    mft.OTF = otf.detach()
    ft = mft(V, F, C)
    img = dm.render_image_from_ftmesh(ft, otf, shape)
    nimg = dm.normalize_tensor(img)
    if str(d["loss_kind"]) == "sum":
        loss = nimg.sum()
    else:
        loss = torch.mean((nimg - _t(d["target"])) ** 2)
    loss.backward()
    band = mft.band().cpu().numpy()
    common, ia, ib = np.intersect1d(band, d["idx"], return_indices=True)
    assert len(common) >= 0.999 * len(d["idx"])
    ftb = ft.detach().reshape(-1).cpu().numpy()[common]
    e_ft = rel_l2(ftb, d["ft"][ib])
    e_img = rel_l2(img.detach().cpu().numpy(), d["image"])
    img_fft = torch.abs(torch.fft.ifftn(ft.detach() * 1 * otf.detach(), list(shape)))
    print(name, "image vs reference float64: %.2e (cuFFT of the same spectrum %.2e)" % (
        e_img, rel_l2(img_fft.cpu().numpy(), d["image"])))
    # the vertex gradient through each combination of render route and normalize
    for route in ("bandbox", "cufft"):
        for nrm in ("kernels", "eager"):
            Vx = _t(d["verts"]).requires_grad_(True)
            ftx = mft(Vx, F, C.detach())
            if route == "cufft":
                ftx = ftx * 1
            ix = dm.render_image_from_ftmesh(ftx, otf.detach(), shape)
            if nrm == "kernels":
                nx = dm.normalize_tensor(ix)
            else:
                nx = (ix - ix.min()) / (ix.max() - ix.min())
            lx = nx.sum() if str(d["loss_kind"]) == "sum" else \
                torch.mean((nx - _t(d["target"])) ** 2)
            lx.backward()
            print(name, route, nrm, "verts %.2e" % rel_l2(Vx.grad.cpu().numpy(), d["grad_verts"]))
    assert e_ft < TOL_FT, name
    assert e_img < TOL_FT, name
    ev = rel_l2(V.grad.cpu().numpy(), d["grad_verts"])
    ec = rel_l2(C.grad.cpu().numpy(), d["grad_coeff"])
    es = rel_l2(S.grad.cpu().numpy(), d["grad_sigma"])
    # the reference's own float32 path is much further away on the vertex gradient
    print(name, "rel-L2 vs reference float64: verts %.2e (reference float32 %.2e) "
          "coeff %.2e (%.2e) sigma %.2e (%.2e)" % (
              ev, rel_l2(d["grad_verts_f32"], d["grad_verts"]),
              ec, rel_l2(d["grad_coeff_f32"], d["grad_coeff"]),
              es, rel_l2(d["grad_sigma_f32"], d["grad_sigma"])))
    assert abs(float(loss.detach()) - float(d["loss"])) < 1e-4 * abs(float(d["loss"])), name
    # Through |.| and normalize_tensor the gradients can be ill-conditioned in the
    # spectrum (d|z|/dz = z/|z| at near-zero voxels, the argmin voxel): the floor
    # is how much the float64 gradients move under a 3e-7 relative perturbation
    # of the spectrum, scaled up when this chain's own spectrum or image is
    # further than that from float64; agreement is required to the larger of the
    # fixed tolerance and twice that floor.
    fl = oracle.chain_floor(d["verts"], d["faces"], d["coeff"], d["box_size"], shape,
                            d["sigma"], float(d["thresh"]), str(d["loss_kind"]), d.get("target"),
                            trials=6)
    k = max(1.0, e_ft / 3e-7, e_img / 3e-7)
    print(name, "conditioning floor", fl, "spectrum %.2e image %.2e: floor x %.2f" % (
        e_ft, e_img, k))
    assert ev < max(TOL_CHAIN_V, 2 * k * fl["verts"]), name
    assert ec < max(TOL_CHAIN, 2 * k * fl["coeff"]), name
    assert es < max(TOL_CHAIN, 2 * k * fl["sigma"]), name


def test_deterministic_bitwise():
    v, f, c, box, shape, sigma, thresh = _case(3, (32, 32, 32), seed=4)
    grid, xi, otf, band = _setup(v, f, c, box, shape, sigma, thresh)
    V, F, C = _t(v), _t(f, torch.int64), _t(c)
    g = torch.randn(band.numel(), dtype=torch.complex64, device=DEV)
    outs = []
    for _ in range(2):
        ft = ops.meshft_list(V, F, C, grid, band)
        gv, gc, _ = ops.meshft_backward_list(V, F, C, grid, band, ft, grad_list=g)
        outs.append((ft.clone(), gv.clone(), gc.clone()))
    for a, b in zip(outs[0], outs[1]):
        assert torch.equal(a, b)


def test_empty_band_and_tiny_meshes():
    v, f, c, box, shape, sigma, thresh = _case(1, (12, 12, 12))
    grid, xi, otf, _ = _setup(v, f, c, box, shape, sigma, thresh)
    V, F, C = _t(v), _t(f, torch.int64), _t(c)
    empty = ops.narrowband(otf, 2.0)
    assert empty.numel() == 0
    ft = ops.meshft_list(V, F, C, grid, empty)
    assert ft.numel() == 0
    gv, gc, _ = ops.meshft_backward_list(V, F, C, grid, empty, ft,
                                         grad_list=torch.zeros(0, dtype=torch.complex64,
                                                               device=DEV))
    assert torch.count_nonzero(gv) == 0 and torch.count_nonzero(gc) == 0
    # a single face
    band = ops.narrowband(otf, 1e-5)
    ft1 = ops.meshft_list(V, F[:1].contiguous(), C[:1].contiguous(), grid, band)
    xil = _oracle_xi(grid, band)
    ref = oracle.meshft_forward(v - box[:, 0], f[:1], c[:1], xil)
    assert rel_l2(ft1.cpu().numpy(), ref) < TOL_FT


def test_bad_face_index_raises():
    v, f, c, box, shape, sigma, thresh = _case(1, (12, 12, 12))
    grid, xi, otf, band = _setup(v, f, c, box, shape, sigma, thresh)
    V, C = _t(v), _t(c)
    fbad = f.copy()
    fbad[3, 1] = len(v) + 5
    F = _t(fbad, torch.int64)
    ft = ops.meshft_list(V, F, C, grid, band)  # forward clamps and flags
    with pytest.raises(IndexError):
        ops.meshft_backward_list(V, F, C, grid, band, ft,
                                 grad_list=torch.ones(band.numel(), dtype=torch.complex64,
                                                      device=DEV))


def test_degenerate_cube_on_odd_grid():
    d = load_golden("cube_degenerate")
    shape = tuple(int(s) for s in d["box_shape"])
    grid, xi, otf, band = _setup(d["verts"], d["faces"], d["coeff"], d["box_size"], shape,
                                 d["sigma"], float(d["thresh"]))
    V, F, C = _t(d["verts"]), _t(d["faces"], torch.int64), _t(d["coeff"])
    ft = ops.meshft_list(V, F, C, grid, band)
    xil = _oracle_xi(grid, band)
    vs = d["verts"] - d["box_size"][:, 0]
    ref = oracle.meshft_forward(vs, d["faces"], d["coeff"], xil)
    assert rel_l2(ft.cpu().numpy(), ref) < TOL_FT
    # xi = 0 is on the odd grid: ft(0) = 1
    k0 = np.ravel_multi_index(tuple(s // 2 for s in shape), shape)
    pos = np.searchsorted(band.cpu().numpy(), k0)
    assert abs(complex(ft[pos].cpu()) - 1.0) < 1e-6
    g = np.exp(1j * np.arange(band.numel()) * 0.1) * otf.reshape(-1)[band.long()].cpu().numpy()
    gv, gc, _ = ops.meshft_backward_list(V, F, C, grid, band, ft,
                                         grad_list=_t(g, torch.complex64))
    rv, rc = oracle.meshft_backward(vs, d["faces"], d["coeff"], xil, g, ref)
    assert rel_l2(gv.cpu().numpy(), rv) < TOL_GV
    assert rel_l2(gc.cpu().numpy(), rc) < TOL_GC


def test_full_size_properties_200cube_20480_faces():
    """Size-independent checks at the fit configuration (200^3, level-5 SH shape):
    translation -> phase, Faces_coeff scale invariance, and oracle agreement on a
    random subsample of the band."""
    v, f = random_sh_shape(5, 0.3, 6, 0.08, seed=11)
    box = oracle.compute_box_size(v, 0.2)
    shape = (200, 200, 200)
    grid, xi, otf, band = _setup(v, f, np.ones(len(f)), box, shape,
                                 np.diag([1e-3, 1e-3, 4e-3]), 1e-5)
    assert 10000 < band.numel() < 20000
    V, F = _t(v), _t(f, torch.int64)
    C = torch.ones(len(f), device=DEV)
    ft = ops.meshft_list(V, F, C, grid, band)
    ft2 = ops.meshft_list(V, F, C * 3.7, grid, band)
    assert rel_l2(ft2.cpu().numpy(), ft.cpu().numpy()) < 2e-6
    t = np.array([0.011, -0.007, 0.003])
    ftt = ops.meshft_list(_t(v + t), F, C, grid, band)
    xil = _oracle_xi(grid, band)
    pred = ft.cpu().numpy() * np.exp(-1j * xil @ t)
    assert rel_l2(ftt.cpu().numpy(), pred) < 1e-5
    rng = np.random.default_rng(0)
    sub = np.sort(rng.choice(band.numel(), 256, replace=False))
    ref = oracle.meshft_forward(v - box[:, 0], f, np.ones(len(f)), xil[sub])
    assert rel_l2(ft.cpu().numpy()[sub], ref) < TOL_FT


def test_device_status_word_reports_bad_band_index():
    """A band index outside the grid (injected on the host) is skipped by the
    kernels and reported through the workspace status word, not a fault."""
    import ctypes
    from deltamic_b200 import _native as N
    v, f, c, box, shape, sigma, thresh = _case(1, (12, 12, 12))
    grid, xi, otf, band = _setup(v, f, c, box, shape, sigma, thresh)
    lib = N.lib()
    bad = band.clone()
    bad[5] = 12 ** 3 + 100
    V, F, C = _t(v), _t(f, torch.int64), _t(c)
    nb = bad.numel()
    ws = torch.zeros(lib.dm_meshft_forward_workspace_size(len(v), len(f), nb), dtype=torch.uint8,
                     device=DEV)
    ft = torch.empty(nb, dtype=torch.complex64, device=DEV)
    spec = torch.zeros(shape, dtype=torch.complex64, device=DEV)
    st = lib.dm_meshft_forward(N.ptr(V), len(v), N.ptr(F), len(f), N.ptr(C),
                               ctypes.byref(grid.cbox), N.ptr(bad), nb, None, N.ptr(ft),
                               N.ptr(spec), N.ptr(ws), ws.numel(), N.stream_ptr(DEV))
    assert st == N.DM_OK
    flags = N._INT()
    assert lib.dm_device_error(N.ptr(ws), ctypes.byref(flags), N.stream_ptr(DEV)) == N.DM_OK
    assert flags.value & N.DM_ERR_BAD_INDEX
    assert lib.dm_device_error(N.ptr(ws), ctypes.byref(flags), N.stream_ptr(DEV)) == N.DM_OK
    assert flags.value == 0  # cleared by the read


def test_float64_module_runs_float64_kernels():
    """dtype=float64 runs the float64 kernels: its spectrum matches the float64
    oracle far below the float32 path's error (tests/test_gpu_float64.py holds
    the tight checks)."""
    import deltamic_b200 as dm
    v, f, c, box, shape, sigma, thresh = _case(2, (20, 20, 20))
    out = []
    for dt in (torch.float32, torch.float64):
        V = torch.tensor(v, dtype=dt, device=DEV, requires_grad=True)
        C = torch.tensor(c, dtype=dt, device=DEV)
        m = dm.Fourier3dMesh(torch.tensor(box), shape, device=DEV, dtype=dt,
                             narrowband_thresh=thresh)
        S = torch.tensor(sigma, dtype=dt, device=DEV)
        m.OTF = dm.generate_gaussian_psf(S, m.xi0, m.xi1, m.xi2)
        ft = m(V, _t(f, torch.int64), C)
        ft.abs().sum().backward()
        out.append((ft.detach().cpu().numpy(), V.grad.cpu().numpy(), m.band().cpu().numpy()))
        assert ft.dtype == (torch.complex64 if dt == torch.float32 else torch.complex128)
    idx = out[1][2].astype(np.int64)
    xil = oracle.xi_list_from_band(idx, oracle.frequency_axes(box, shape))
    ref = oracle.meshft_forward(v - box[:, 0], f, c, xil, seps=oracle.SEPS_F32)
    assert rel_l2(out[1][0].reshape(-1)[idx], ref) < 1e-11
    assert rel_l2(out[0][0].reshape(-1)[idx], ref) < TOL_FT
    assert rel_l2(out[1][1], out[0][1]) < 1e-5


@pytest.mark.parametrize("level,shape", [(2, (24, 20, 18)), (2, (15, 17, 13)), (3, (32, 31, 30))])
def test_half_band_matches_full_band(level, shape):
    """A band from a Gaussian OTF is mirror-symmetric, so the kernels evaluate
    half of it; the results equal the every-frequency path (a clone of the band
    carries no symmetry flag) and the oracle.  Odd shapes hold xi = 0 itself."""
    v, f, c, box, shape, sigma, thresh = _case(level, shape, sigma=np.array(
        [[2e-3, 4e-4, 0.0], [4e-4, 1e-3, -3e-4], [0.0, -3e-4, 4e-3]]))
    grid, xi, otf, band = _setup(v, f, c, box, shape, sigma, thresh)
    assert ops.band_is_hermitian(band)
    full = band.clone()
    assert not ops.band_is_hermitian(full)
    V, F, C = _t(v), _t(f, torch.int64), _t(c)
    ft_h = ops.meshft_list(V, F, C, grid, band)
    ft_g = ops.meshft_list(V, F, C, grid, full)
    h = ft_h.cpu().numpy()
    assert np.array_equal(h[::-1], np.conj(h))
    assert rel_l2(h, ft_g.cpu().numpy()) < 1e-6
    ref = oracle.meshft_forward(v - box[:, 0], f, c, _oracle_xi(grid, band))
    assert rel_l2(h, ref) < TOL_FT
    rng = np.random.default_rng(5)
    G = _t(rng.normal(size=(band.numel(), 2))).view(torch.complex64).view(-1).contiguous()
    oh = ops.meshft_backward_list(V, F, C, grid, band, ft_h, grad_list=G, otf=otf.view(-1),
                                  want_otf=True)
    og = ops.meshft_backward_list(V, F, C, grid, full, ft_g, grad_list=G, otf=otf.view(-1),
                                  want_otf=True)
    for a, b in zip(oh, og):
        assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-5
    gv_ref, gc_ref = oracle.meshft_backward(
        v - box[:, 0], f, c, _oracle_xi(grid, band),
        (G * otf.view(-1)[band.long()]).cpu().numpy().astype(np.complex128), ref)
    assert rel_l2(oh[0].cpu().numpy(), gv_ref) < TOL_GV
    assert rel_l2(oh[1].cpu().numpy(), gc_ref) < TOL_GC


def test_asymmetric_band_takes_the_full_path():
    v, f, c, box, shape, sigma, thresh = _case(2, (20, 20, 20))
    grid, xi, otf, band = _setup(v, f, c, box, shape, sigma, thresh)
    o2 = otf.clone().view(-1)
    o2[band[:3].long()] = 0.0  # drop three voxels on one side only
    b2 = ops.narrowband(o2.view(otf.shape), thresh)
    assert not ops.band_is_hermitian(b2)
    ft = ops.meshft_list(_t(v), _t(f, torch.int64), _t(c), grid, b2)
    ref = oracle.meshft_forward(v - box[:, 0], f, c, _oracle_xi(grid, b2))
    assert rel_l2(ft.cpu().numpy(), ref) < TOL_FT


def test_symmetry_flag_on_asymmetric_band_is_reported():
    """DM_BAND_HERMITIAN on a band that is not mirror-symmetric is caught by the
    kernels' mirror check (status word), with every access in bounds."""
    import ctypes
    from deltamic_b200 import _native as N
    v, f, c, box, shape, sigma, thresh = _case(1, (12, 12, 12))
    grid, xi, otf, band = _setup(v, f, c, box, shape, sigma, thresh)
    bad = band[1:].contiguous()  # one entry short: the mirror relation breaks
    lib = N.lib()
    V, F, C = _t(v), _t(f, torch.int64), _t(c)
    nb = bad.numel()
    ws = torch.zeros(lib.dm_meshft_forward_workspace_size(len(v), len(f), nb), dtype=torch.uint8,
                     device=DEV)
    ft = torch.empty(nb, dtype=torch.complex64, device=DEV)
    box_h = ops.band_box(grid, True)
    st = lib.dm_meshft_forward(N.ptr(V), len(v), N.ptr(F), len(f), N.ptr(C), ctypes.byref(box_h),
                               N.ptr(bad), nb, None, N.ptr(ft), None, N.ptr(ws), ws.numel(),
                               N.stream_ptr(DEV))
    assert st == N.DM_OK
    flags = N._INT()
    assert lib.dm_device_error(N.ptr(ws), ctypes.byref(flags), N.stream_ptr(DEV)) == N.DM_OK
    assert flags.value & N.DM_ERR_BAD_INDEX


def test_every_tile_variant_matches_oracle():
    """Each forward and adjoint tile-shape variant (the autotuner's candidates,
    including the paired-FP32 two-frequency forward and two-face adjoint) against
    the oracle, on a mesh whose pairs take the series, pivot and degenerate paths."""
    import ctypes
    from deltamic_b200 import _native as N
    lib = N.lib()
    v, f, c, box, shape, sigma, thresh = _case(3, (41, 37, 33), seed=6)
    grid, xi, otf, band = _setup(v, f, c, box, shape, sigma, thresh)
    V, F, C = _t(v), _t(f, torch.int64), _t(c)
    xil = _oracle_xi(grid, band)
    ft64 = oracle.meshft_forward(v - box[:, 0], f, c, xil)
    rng = np.random.default_rng(3)
    g = (rng.normal(size=band.numel()) + 1j * rng.normal(size=band.numel())).astype(np.complex64)
    rv, rc = oracle.meshft_backward(v - box[:, 0], f, c, xil, g, ft64)
    fwd, bwd, nf, nb = N._INT(), N._INT(), N._INT(), N._INT()
    N.check(lib.dm_get_variants(ctypes.byref(fwd), ctypes.byref(bwd), ctypes.byref(nf),
                                ctypes.byref(nb)), "dm_get_variants")
    try:
        for k in range(max(nf.value, nb.value)):
            N.check(lib.dm_set_variants(min(k, nf.value - 1), min(k, nb.value - 1)),
                    "dm_set_variants")
            ft = ops.meshft_list(V, F, C, grid, band)
            gv, gc, _ = ops.meshft_backward_list(V, F, C, grid, band, ft,
                                                 grad_list=_t(g, torch.complex64))
            e = (rel_l2(ft.cpu().numpy(), ft64), rel_l2(gv.cpu().numpy(), rv),
                 rel_l2(gc.cpu().numpy(), rc))
            print(f"variant {k}: ft {e[0]:.2e} verts {e[1]:.2e} coeff {e[2]:.2e}")
            assert e[0] < TOL_FT and e[1] < TOL_GV and e[2] < TOL_GC, k
    finally:
        lib.dm_set_variants(fwd.value, bwd.value)
