"""The oracle against the reference's own outputs at the benchmark configurations
(golden vectors made by tests/golden/make_golden_configs.py from deltamic's
MeshFTPy + torch autograd).

cfg1 (level-3 icosphere, 64^3, sum of the normalised image) is checked end to end
(spectrum, image samples, loss, gradients to Verts, Faces_coeff and sigma); cfg4
(level-4 SH mesh, 128^3, image L2) on a 1,024-frequency sample of its spectrum
(the whole chain there is 1.3e8 pairs per pass, minutes of numpy)."""
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN_DIR, load_golden, rel_l2


def _have(name):
    return os.path.exists(os.path.join(GOLDEN_DIR, name + ".npz"))


@pytest.mark.skipif(not _have("cfg1_icosphere_l3_64"), reason="golden not generated")
def test_oracle_matches_reference_cfg1():
    d = load_golden("cfg1_icosphere_l3_64")
    o = oracle.pipeline(d["verts"], d["faces"], d["coeff"], d["box_size"], d["box_shape"],
                        d["sigma"], float(d["thresh"]), loss=str(d["loss_kind"]))
    assert np.array_equal(o["idx"], d["idx"])
    assert rel_l2(o["ft"], d["ft"]) < 1e-11
    img = o["image"].reshape(-1)
    assert rel_l2(img[d["image_sample_idx"]], d["image_sample"]) < 1e-11
    assert abs(img.sum() - float(d["image_sum"])) < 1e-10 * abs(float(d["image_sum"]))
    assert abs(o["loss"] - float(d["loss"])) <= 1e-10 * abs(float(d["loss"]))
    assert rel_l2(o["grad_verts"], d["grad_verts"]) < 1e-7
    assert rel_l2(o["grad_coeff"], d["grad_coeff"]) < 1e-10
    assert rel_l2(o["grad_sigma"], d["grad_sigma"]) < 1e-10
    # the reference's own float32 run, for the record: its vertex gradient is far
    # from float64, its spectrum close
    assert rel_l2(d["ft_f32"], d["ft"]) < 1e-4


@pytest.mark.skipif(not _have("cfg4_sh_l4_128"), reason="golden not generated")
def test_oracle_matches_reference_cfg4_spectrum_sample():
    d = load_golden("cfg4_sh_l4_128")
    axes = oracle.frequency_axes(d["box_size"], d["box_shape"])
    otf = oracle.gaussian_otf(d["sigma"], *axes)
    idx = oracle.band_indices(otf, float(d["thresh"]))
    assert np.array_equal(idx, d["idx"])
    sub = np.sort(np.random.default_rng(0).choice(len(idx), 1024, replace=False))
    xi = oracle.xi_list_from_band(idx[sub], axes)
    ft = oracle.meshft_forward(d["verts"] - d["box_size"][:, 0], d["faces"], d["coeff"], xi)
    # the sampled entries of (2/M) sum_k A_k c_k F_k, M over all faces
    assert rel_l2(ft, d["ft"][sub]) < 1e-11
    t = oracle.smooth_target(tuple(int(s) for s in d["box_shape"]), int(d["target_seed"]))
    assert t.shape == tuple(int(s) for s in d["box_shape"])
