"""The convolution oracle against torch's own conv3d on CPU (float64)."""
import numpy as np
import torch

from oracle.conv import conv_backward, conv_forward


def test_conv_oracle_matches_torch_conv3d():
    rng = np.random.default_rng(0)
    B, D, H, W, Ci, Co = 2, 9, 8, 7, 3, 4
    x = rng.normal(size=(B, D, H, W, Ci))
    w = rng.normal(size=(27 * Ci, Co)) * 0.2
    b = rng.normal(size=Co)
    pre, act = conv_forward(x, w, b)
    dact = rng.normal(size=act.shape)
    dx, dw, db = conv_backward(x, w, pre, dact)

    xt = torch.tensor(x).permute(0, 4, 1, 2, 3).requires_grad_(True)
    wt = torch.tensor(w.reshape(3, 3, 3, Ci, Co)).permute(4, 3, 0, 1, 2).requires_grad_(True)
    bt = torch.tensor(b).requires_grad_(True)
    pt = torch.nn.functional.conv3d(xt, wt, bt, stride=2, padding=1)
    at = torch.nn.functional.gelu(pt)
    at.backward(torch.tensor(dact).permute(0, 4, 1, 2, 3))
    assert np.allclose(pre, pt.detach().permute(0, 2, 3, 4, 1).numpy(), atol=1e-12)
    assert np.allclose(act, at.detach().permute(0, 2, 3, 4, 1).numpy(), atol=1e-12)
    assert np.allclose(dx, xt.grad.permute(0, 2, 3, 4, 1).numpy(), atol=1e-10)
    assert np.allclose(dw, wt.grad.permute(2, 3, 4, 1, 0).reshape(27 * Ci, Co).numpy(), atol=1e-10)
    assert np.allclose(db, bt.grad.numpy(), atol=1e-10)
