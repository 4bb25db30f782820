"""Learned initialiser: a small 3D-conv encoder that maps a rendered 64^3 image to
per-vertex displacements of a level-4 icosphere template, giving the fitting loop
a starting mesh closer than the sphere (no counterpart in the reference).

Network: four 3x3x3 stride-2 convolutions 1 -> 16 -> 32 -> 64 -> 128 with GELU
(BF16 implicit GEMMs of ``csrc/conv.cu`` on tcgen05 tensor cores, FP32
accumulators in tensor memory), global
average pooling, then an MLP 128 -> 512 (GELU) -> 2,562 x 3.  Training pairs are
rendered by this package's own renderer (``BatchRenderer``) from random
spherical-harmonic shapes with random anisotropic Gaussian PSFs and
Poisson + read noise.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch
from torch import nn

from . import _native as N
from .batch import BatchRenderer
from .mesh import icosphere, real_sph_harm

__all__ = ["LearnedInit", "conv3d_s2", "conv_status_check", "ShapeSampler", "render_batch",
           "train_learned_init", "save_checkpoint", "load_checkpoint"]

CHANNELS = (1, 16, 32, 64, 128)
IMAGE = 64
BOX = np.array([[-0.5, 0.5]] * 3)
TEMPLATE_LEVEL = 4


def _kp(ci):
    return (27 * ci + 31) // 32 * 32


class _ConvS2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, w32, b32):
        lib = N.lib()
        B, D, H, W, Ci = x.shape
        Kp, Co = w32.shape
        wb = w32.to(torch.bfloat16).contiguous()
        Do, Ho, Wo = (D + 1) // 2, (H + 1) // 2, (W + 1) // 2
        pre = torch.empty(B, Do, Ho, Wo, Co, dtype=torch.float32, device=x.device)
        act = torch.empty(B, Do, Ho, Wo, Co, dtype=torch.bfloat16, device=x.device)
        ws = N.WORKSPACES.get(("conv_fwd", Ci, Co),
                              lib.dm_conv3d_s2_forward_workspace_size(B, D, H, W, Ci, Co),
                              x.device)
        N.check(lib.dm_conv3d_s2_forward_ws(N.ptr(x), B, D, H, W, Ci, N.ptr(wb), N.ptr(b32), Co,
                                            N.ptr(pre), N.ptr(act), N.ptr(ws), ws.numel(),
                                            N.stream_ptr(x.device)), "dm_conv3d_s2_forward_ws")
        ctx.save_for_backward(x, wb, pre)
        return act

    @staticmethod
    def backward(ctx, dact):
        lib = N.lib()
        x, wb, pre = ctx.saved_tensors
        B, D, H, W, Ci = x.shape
        Kp, Co = wb.shape
        dact = dact.to(torch.bfloat16).contiguous()
        dx = torch.empty(x.shape, dtype=torch.bfloat16, device=x.device) \
            if ctx.needs_input_grad[0] else None
        dw = torch.empty(Kp, Co, dtype=torch.float32, device=x.device)
        db = torch.empty(Co, dtype=torch.float32, device=x.device)
        ws = N.WORKSPACES.get(("conv", Ci, Co),
                              lib.dm_conv3d_s2_workspace_size(B, D, H, W, Ci, Co), x.device)
        N.check(lib.dm_conv3d_s2_backward_bf16(N.ptr(x), B, D, H, W, Ci, N.ptr(wb), Co,
                                               N.ptr(pre), N.ptr(dact), N.ptr(dx), N.ptr(dw),
                                               N.ptr(db), N.ptr(ws), ws.numel(),
                                               N.stream_ptr(x.device)),
                "dm_conv3d_s2_backward_bf16")
        return dx, dw, db


def conv_status_check(device):
    """Raise if a convolution kernel gave up a bounded wait since the last check
    (reads and clears the kernels' status word; synchronises ``device``'s stream)."""
    flags = ctypes.c_int(0)
    N.check(N.lib().dm_conv3d_s2_device_error(ctypes.byref(flags), N.stream_ptr(device)),
            "dm_conv3d_s2_device_error")
    N.check(flags.value, "convolution kernels")


def conv3d_s2(x, w32, b32):
    """GELU(conv3d(x, w, stride 2, padding 1) + b), channels-last BF16 in and out."""
    N.require_cuda(x, "x", torch.bfloat16)
    return _ConvS2.apply(x.contiguous(), w32, b32)


class LearnedInit(nn.Module):
    def __init__(self, n_verts=None, hidden=512, seed=0):
        super().__init__()
        if n_verts is None:
            n_verts = len(icosphere(TEMPLATE_LEVEL)[0])
        g = torch.Generator().manual_seed(seed)
        self.w = nn.ParameterList()
        self.b = nn.ParameterList()
        for ci, co in zip(CHANNELS[:-1], CHANNELS[1:]):
            w = torch.zeros(_kp(ci), co)
            w[:27 * ci] = torch.randn(27 * ci, co, generator=g) * math.sqrt(2.0 / (27 * ci))
            self.w.append(nn.Parameter(w))
            self.b.append(nn.Parameter(torch.zeros(co)))
        self.fc1 = nn.Linear(CHANNELS[-1], hidden)
        self.fc2 = nn.Linear(hidden, 3 * n_verts)
        with torch.no_grad():
            self.fc2.weight.mul_(0.01)
            self.fc2.bias.zero_()
        self.n_verts = n_verts

    def encode(self, img):
        """img [B, D, H, W] float -> pooled features [B, 128]."""
        x = img.to(torch.bfloat16).unsqueeze(-1).contiguous()
        for w, b in zip(self.w, self.b):
            x = conv3d_s2(x, w, b)
        return x.float().mean(dim=(1, 2, 3))

    def forward(self, img):
        """Per-vertex displacements [B, n_verts, 3] of the template."""
        h = torch.nn.functional.gelu(self.fc1(self.encode(img)))
        return self.fc2(h).view(img.shape[0], self.n_verts, 3)


class ShapeSampler:
    """Random radial SH shapes r = r0 (1 + sum_{l<=lmax} a_lm Y_lm), a_lm ~ N(0, (amp/l)^2)
    on the level-4 template, with anisotropic Gaussian PSFs diag U[5e-4, 4e-3]."""

    def __init__(self, r0=0.3, lmax=8, amp=0.1, level=TEMPLATE_LEVEL):
        self.r0, self.lmax, self.amp = r0, lmax, amp
        self.template, self.faces = icosphere(level, r0)
        d = self.template / np.linalg.norm(self.template, axis=1, keepdims=True)
        th = np.arccos(np.clip(d[:, 2], -1, 1))
        ph = np.arctan2(d[:, 1], d[:, 0])
        self.dirs = d
        self.lm = [(l, m) for l in range(1, lmax + 1) for m in range(-l, l + 1)]
        self.Y = np.stack([real_sph_harm(l, m, th, ph) for l, m in self.lm], 1)  # [nv, n_lm]
        self.sd = np.array([amp / l for l, m in self.lm])

    def sample(self, n, rng):
        a = rng.normal(size=(n, len(self.lm))) * self.sd
        r = self.r0 * (1.0 + a @ self.Y.T)                    # [n, nv]
        verts = self.dirs[None] * r[..., None]                 # [n, nv, 3]
        sig = rng.uniform(5e-4, 4e-3, size=(n, 3))
        return verts, sig


def render_batch(verts, sig, faces, rng_seed, device, thresh=1e-5, photons=200.0,
                 read_noise=2.0):
    """Noisy 64^3 images of ``verts[n, nv, 3]`` (one BatchRenderer launch set).

    Returns ``(inputs, targets)``: the min/max-normalised noisy images (network
    input) and the noisy images divided by the ``photons`` exposure (fit target,
    unbiased against the min/max-normalised render)."""
    n = len(verts)
    br = BatchRenderer([BOX] * n, [(IMAGE,) * 3] * n, thresh, device)
    br.set_sigmas([np.diag(s) for s in sig])
    br.set_meshes(list(verts), [faces] * n)
    V = torch.tensor(np.concatenate(verts), dtype=torch.float32, device=device)
    C = torch.ones(n * len(faces), device=device)
    img = br.render(V, C).view(n, IMAGE, IMAGE, IMAGE)
    gen = torch.Generator(device=device).manual_seed(int(rng_seed))
    mx = img.amax(dim=(1, 2, 3), keepdim=True)
    ph = img / mx * photons
    noisy = torch.poisson(ph, generator=gen) + read_noise * torch.randn(
        img.shape, device=device, generator=gen)
    lo = noisy.amin(dim=(1, 2, 3), keepdim=True)
    hi = noisy.amax(dim=(1, 2, 3), keepdim=True)
    return (noisy - lo) / (hi - lo), noisy / photons


def train_learned_init(n_train, epochs, batch=64, lr=1e-3, seed=0, device="cuda",
                       model=None, log=None):
    """Render ``n_train`` pairs with the package's renderer, then train with Adam
    (cosine-decayed learning rate) on the vertex-position MSE.  Returns (model,
    sampler, per-epoch losses)."""
    rng = np.random.default_rng(seed)
    sampler = ShapeSampler()
    imgs, disps = [], []
    tmpl = torch.tensor(sampler.template, dtype=torch.float32, device=device)
    for s in range(0, n_train, batch):
        k = min(batch, n_train - s)
        v, sig = sampler.sample(k, rng)
        imgs.append(render_batch(v, sig, sampler.faces, rng.integers(1 << 30), device)[0]
                    .to(torch.bfloat16))
        disps.append(torch.tensor(v, dtype=torch.float32, device=device) - tmpl)
    imgs = torch.cat(imgs)
    disps = torch.cat(disps)
    model = (model or LearnedInit(len(sampler.template), seed=seed)).to(device)
    opt = torch.optim.Adam(model.parameters(), lr=lr)
    iters = epochs * ((n_train + batch - 1) // batch)
    sched = torch.optim.lr_scheduler.LambdaLR(
        opt, lambda it: 0.5 * (1.0 + math.cos(math.pi * min(it, iters) / max(iters, 1))))
    g = torch.Generator(device=device).manual_seed(seed)
    hist = []
    for ep in range(epochs):
        perm = torch.randperm(n_train, device=device, generator=g)
        tot = torch.zeros((), device=device)
        for s in range(0, n_train, batch):
            idx = perm[s:s + batch]
            pred = model(imgs[idx].float())
            loss = torch.mean((pred - disps[idx]) ** 2)
            opt.zero_grad(set_to_none=True)
            loss.backward()
            opt.step()
            sched.step()
            tot += loss.detach() * len(idx)
        hist.append(float(tot) / n_train)
        conv_status_check(torch.device(device))
        if log:
            log(f"epoch {ep}: vertex MSE {hist[-1]:.3e}")
    return model, sampler, hist


def evaluate_learned_init(model, sampler, n_eval=256, steps=300, lr=1e-3, seed=12345,
                          device="cuda", chunk=64, tol=0.01):
    """Held-out comparison of learned-init + GD against sphere-init GD.

    For every shape both fits run ``steps`` Adam steps on the image L2 (cells of a
    chunk are fitted together, each with its own loss).  The plain fit's final
    loss L_p is the target; the learned fit's time to reach (1 + tol) L_p counts
    the network inference plus its steps.  Returns per-shape arrays and timings.
    """
    from .batch import BatchFitStep
    from .ops import FreqGrid, iou, voxelize
    rng = np.random.default_rng(seed)
    tmpl = torch.tensor(sampler.template, dtype=torch.float32, device=device)
    faces_t = torch.tensor(sampler.faces, device=device)
    grid = FreqGrid(BOX, (IMAGE,) * 3)
    out = {k: [] for k in ("plain_final", "learned_first", "learned_steps", "reached",
                           "iou_plain", "iou_learned", "iou_learned_init", "iou_sphere",
                           "iou_learned_at_target")}
    t_step = t_infer = 0.0
    n_steps_timed = n_infer = 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for s0 in range(0, n_eval, chunk):
        k = min(chunk, n_eval - s0)
        v, sig = sampler.sample(k, rng)
        net_in, target = render_batch(v, sig, sampler.faces, rng.integers(1 << 30), device)
        br = BatchRenderer([BOX] * k, [(IMAGE,) * 3] * k, 1e-5, device)
        br.set_sigmas([np.diag(x) for x in sig])
        br.set_meshes([sampler.template] * k, [sampler.faces] * k)
        C = torch.ones(k * len(sampler.faces), device=device)
        tgt = target.reshape(-1).contiguous()
        # learned initial meshes (inference timed)
        torch.cuda.synchronize()
        e0.record()
        with torch.no_grad():
            init_l = (model(net_in) + tmpl).reshape(-1, 3).contiguous()
        e1.record()
        torch.cuda.synchronize()
        t_infer += e0.elapsed_time(e1)
        n_infer += k
        curves = {}
        snaps = {}
        for name, V0 in (("plain", tmpl.repeat(k, 1)), ("learned", init_l)):
            st = BatchFitStep(br, V0.clone(), C, tgt, "mse", 0.0, lr, graph=True)
            losses = torch.zeros(steps, k, device=device)
            hist = [] if name == "learned" else None
            torch.cuda.synchronize()
            e0.record()
            for i in range(steps):
                st()
                losses[i] = st.cell_losses
                if hist is not None and i % 10 == 9:
                    hist.append(st.V.detach().clone())
            e1.record()
            torch.cuda.synchronize()
            t_step += e0.elapsed_time(e1)
            n_steps_timed += steps * k
            curves[name] = (losses.cpu().numpy(), st.V.view(k, -1, 3))
            snaps[name] = hist
        lp, Vp = curves["plain"]
        ll, Vl = curves["learned"]
        target_l2 = lp[-1] * (1 + tol)
        gt = torch.tensor(v, dtype=torch.float32, device=device)
        V0l = init_l.view(k, -1, 3)
        for c in range(k):
            hit = np.flatnonzero(ll[:, c] <= target_l2[c])
            out["plain_final"].append(float(lp[-1, c]))
            out["learned_first"].append(float(ll[0, c]))
            n_hit = int(hit[0]) + 1 if len(hit) else steps
            out["learned_steps"].append(n_hit)
            out["reached"].append(bool(len(hit)))
            occ_gt = voxelize(gt[c].contiguous(), faces_t, grid)
            occ = lambda VV: iou(voxelize(VV.contiguous(), faces_t, grid), occ_gt)
            out["iou_plain"].append(occ(Vp[c]))
            out["iou_learned"].append(occ(Vl[c]))
            out["iou_learned_init"].append(occ(V0l[c]))
            out["iou_sphere"].append(occ(tmpl))
            # mesh at the reach step, from the snapshots taken every 10 steps
            j = min(max((n_hit + 9) // 10 - 1, 0), len(snaps["learned"]) - 1)
            Vs = snaps["learned"][j].view(k, -1, 3)[c] if n_hit > 1 else V0l[c]
            out["iou_learned_at_target"].append(occ(Vs))
    res = {k: np.array(v) for k, v in out.items() if v}
    ms_step = t_step / n_steps_timed      # per shape per step
    ms_infer = t_infer / n_infer          # per shape
    t_plain = steps * ms_step
    t_learned = res["learned_steps"] * ms_step + ms_infer
    res.update(ms_step_per_shape=ms_step, ms_infer_per_shape=ms_infer,
               time_ratio=t_learned / t_plain, steps=steps)
    return res


def save_checkpoint(path, model: LearnedInit, optimizer=None, scheduler=None, **extra) -> None:
    """torch.save of the network (weights, n_verts), the optimiser and scheduler
    states when given, and ``extra`` (epoch, losses, ...)."""
    state = {"model": model.state_dict(), "n_verts": int(model.n_verts),
             "hidden": int(model.fc1.out_features), "extra": dict(extra)}
    if optimizer is not None:
        state["optimizer"] = optimizer.state_dict()
    if scheduler is not None:
        state["scheduler"] = scheduler.state_dict()
    torch.save(state, path)


def load_checkpoint(path, model: LearnedInit = None, optimizer=None, scheduler=None,
                    device=None):
    """Read a file of :func:`save_checkpoint` into ``model`` (a new LearnedInit of
    the saved size when None, on ``device``) and the optimiser / scheduler when
    given; returns ``(model, extra)``."""
    state = torch.load(path, map_location="cpu", weights_only=False)
    if model is None:
        model = LearnedInit(n_verts=state["n_verts"], hidden=state["hidden"])
    model.load_state_dict(state["model"])
    if device is not None:
        model = model.to(device)
    if optimizer is not None and "optimizer" in state:
        optimizer.load_state_dict(state["optimizer"])
    if scheduler is not None and "scheduler" in state:
        scheduler.load_state_dict(state["scheduler"])
    return model, state["extra"]
