"""Learned initialiser: BF16 tensor-core convolutions against the float64 conv
oracle, network gradients against a float32 PyTorch reference, and the gain of
the trained network over the sphere initialisation."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle.conv import conv_backward, conv_forward

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _bf(a):
    return torch.tensor(a, dtype=torch.float32).to(torch.bfloat16)


@pytest.mark.parametrize("shape", [(2, 16, 16, 16, 1, 16), (2, 12, 10, 14, 16, 32),
                                   (1, 8, 8, 8, 32, 64), (2, 6, 6, 6, 64, 128),
                                   (3, 17, 15, 19, 8, 32), (1, 9, 7, 5, 128, 16),
                                   (2, 17, 23, 70, 1, 32), (1, 9, 11, 13, 1, 16),
                                   (3, 8, 8, 8, 64, 128), (1, 9, 7, 14, 32, 64)])
def test_conv_kernels_match_oracle(shape):
    """Forward, weight, bias and data gradients of the tcgen05 implicit GEMMs (and
    of the direct single-channel kernels, Ci = 1) against the float64 oracle on the
    same BF16 inputs (odd extents: ragged row tiles and parity classes; Ci = 8 and
    128: the vector and element gathers; 3 x 8^3 x 64 -> 128: the tap-GEMM kernels with a
    ragged last tile; 1 x 8^3 x 32 -> 64 the persistent tap-GEMM forward and 9 x 7 x 14 x 32
    -> 64 (7 output columns) the footprint forward)."""
    from deltamic_b200.learned import _kp, conv3d_s2, conv_status_check
    B, D, H, W, Ci, Co = shape
    rng = np.random.default_rng(Ci)
    xb = _bf(rng.normal(size=(B, D, H, W, Ci)))
    wpad = np.zeros((_kp(Ci), Co))
    wpad[:27 * Ci] = rng.normal(size=(27 * Ci, Co)) * 0.2
    wb = _bf(wpad)
    b = rng.normal(size=Co) * 0.1
    x = xb.to(DEV).requires_grad_(True)
    w = wb.float().to(DEV).requires_grad_(True)
    bt = torch.tensor(b, dtype=torch.float32, device=DEV).requires_grad_(True)
    act = conv3d_s2(x, w, bt)
    dact = rng.normal(size=act.shape)
    act.backward(torch.tensor(dact, dtype=torch.bfloat16, device=DEV))
    xo, wo = xb.float().numpy(), wb.float().numpy()
    pre, acto = conv_forward(xo, wo, b)
    dx, dw, db = conv_backward(xo, wo, pre, torch.tensor(dact).to(torch.bfloat16).double().numpy())
    assert rel_l2(act.float().detach().cpu().numpy(), acto) < 8e-3
    assert rel_l2(w.grad[:27 * Ci].cpu().numpy(), dw) < 1e-2
    assert rel_l2(bt.grad.cpu().numpy(), db) < 1e-2
    assert rel_l2(x.grad.float().cpu().numpy(), dx) < 1e-2
    conv_status_check(torch.device(DEV))


def test_network_gradients_match_float32_reference():
    from deltamic_b200.learned import CHANNELS, LearnedInit
    torch.manual_seed(0)
    m = LearnedInit(n_verts=162).to(DEV)
    img = torch.rand(2, 32, 32, 32, device=DEV)
    tgt = torch.randn(2, 162, 3, device=DEV) * 0.01
    loss = torch.mean((m(img) - tgt) ** 2)
    loss.backward()

    # float32 reference with the same (bf16-rounded) conv weights
    x = img.to(torch.bfloat16).float().unsqueeze(1)
    ws, bs = [], []
    for (ci, co), w, b in zip(zip(CHANNELS[:-1], CHANNELS[1:]), m.w, m.b):
        wr = w.detach()[:27 * ci].to(torch.bfloat16).float().view(3, 3, 3, ci, co)
        wr = wr.permute(4, 3, 0, 1, 2).contiguous().requires_grad_(True)
        br = b.detach().clone().requires_grad_(True)
        ws.append(wr)
        bs.append(br)
        x = torch.nn.functional.gelu(torch.nn.functional.conv3d(x, wr, br, stride=2, padding=1))
    h = x.mean(dim=(2, 3, 4))
    f1w = m.fc1.weight.detach().clone().requires_grad_(True)
    f2w = m.fc2.weight.detach().clone().requires_grad_(True)
    h = torch.nn.functional.gelu(h @ f1w.T + m.fc1.bias.detach())
    out = (h @ f2w.T + m.fc2.bias.detach()).view(2, 162, 3)
    ref = torch.mean((out - tgt) ** 2)
    ref.backward()
    assert abs(float(loss) - float(ref)) < 2e-2 * abs(float(ref))
    assert rel_l2(m.fc2.weight.grad.cpu().numpy(), f2w.grad.cpu().numpy()) < 3e-2
    for i, (ci, co) in enumerate(zip(CHANNELS[:-1], CHANNELS[1:])):
        g = m.w[i].grad[:27 * ci].view(3, 3, 3, ci, co).permute(4, 3, 0, 1, 2)
        assert rel_l2(g.cpu().numpy(), ws[i].grad.cpu().numpy()) < 5e-2, i
        assert rel_l2(m.b[i].grad.cpu().numpy(), bs[i].grad.cpu().numpy()) < 5e-2, i


@pytest.fixture(scope="module")
def trained():
    """A network trained briefly on 8,192 renderer-generated pairs (12 epochs)."""
    from deltamic_b200.learned import train_learned_init
    model, sampler, hist = train_learned_init(n_train=8192, epochs=12, batch=64, lr=2e-3,
                                              seed=1, device=DEV)
    return model, sampler, hist


def test_trained_network_beats_sphere_initialisation(trained):
    """A briefly trained network predicts held-out shapes far better than the
    template sphere the plain fit starts from."""
    from deltamic_b200.learned import render_batch
    model, sampler, hist = trained
    assert hist[-1] < 0.5 * hist[0]
    rng = np.random.default_rng(999)
    v, sig = sampler.sample(32, rng)
    img, _ = render_batch(v, sig, sampler.faces, 7, DEV)
    with torch.no_grad():
        pred = model(img) + torch.tensor(sampler.template, dtype=torch.float32, device=DEV)
    gt = torch.tensor(v, dtype=torch.float32, device=DEV)
    tmpl = torch.tensor(sampler.template, dtype=torch.float32, device=DEV)
    err_learned = float(torch.sqrt(torch.mean((pred - gt) ** 2)))
    err_sphere = float(torch.sqrt(torch.mean((tmpl - gt) ** 2)))
    print(f"vertex RMSE: learned {err_learned:.4f} sphere {err_sphere:.4f}")
    assert err_learned < 0.7 * err_sphere


def test_learned_init_time_to_fit_and_iou(trained):
    """Held-out shapes: learned init + GD reaches the plain sphere-init fit's final
    image L2 (within 1%) in under a quarter of the plain fit's time (network
    inference included), with a volumetric IoU against the generating mesh of at
    least 0.95 at that point (medians over 32 shapes)."""
    from deltamic_b200.learned import evaluate_learned_init
    model, sampler, _ = trained
    res = evaluate_learned_init(model, sampler, n_eval=32, steps=300, lr=1e-3, seed=4321,
                                device=DEV, chunk=32)
    ratio = float(np.median(res["time_ratio"]))
    iou_t = float(np.median(res["iou_learned_at_target"]))
    print(f"learned init: median time ratio {ratio:.3f} (p90 "
          f"{np.percentile(res['time_ratio'], 90):.3f}), reached {res['reached'].mean():.2f}, "
          f"median IoU at target {iou_t:.3f}, plain final IoU {np.median(res['iou_plain']):.3f}")
    assert res["reached"].mean() >= 0.9
    assert ratio < 0.25
    assert iou_t >= 0.95
