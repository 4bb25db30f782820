"""Learned initialiser: a small 3D-conv encoder that maps a rendered 64^3 image to
per-vertex displacements of a level-4 icosphere template, giving the fitting loop
a starting mesh closer than the sphere (no counterpart in the reference).

Network: four 3x3x3 stride-2 convolutions 1 -> 16 -> 32 -> 64 -> 128 with GELU
(BF16 tensor-core implicit GEMMs of ``csrc/conv.cu``, FP32 accumulation), global
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

__all__ = ["LearnedInit", "conv3d_s2", "ShapeSampler", "render_batch", "train_learned_init"]

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
        N.check(lib.dm_conv3d_s2_forward(N.ptr(x), B, D, H, W, Ci, N.ptr(wb), N.ptr(b32), Co,
                                         N.ptr(pre), N.ptr(act), N.stream_ptr(x.device)),
                "dm_conv3d_s2_forward")
        ctx.save_for_backward(x, wb, pre)
        return act

    @staticmethod
    def backward(ctx, dact):
        lib = N.lib()
        x, wb, pre = ctx.saved_tensors
        B, D, H, W, Ci = x.shape
        Kp, Co = wb.shape
        dact = dact.float().contiguous()
        dx = torch.empty(x.shape, dtype=torch.float32, device=x.device) \
            if ctx.needs_input_grad[0] else None
        dw = torch.empty(Kp, Co, dtype=torch.float32, device=x.device)
        db = torch.empty(Co, dtype=torch.float32, device=x.device)
        ws = N.WORKSPACES.get(("conv", Ci, Co),
                              lib.dm_conv3d_s2_workspace_size(B, D, H, W, Ci, Co), x.device)
        N.check(lib.dm_conv3d_s2_backward(N.ptr(x), B, D, H, W, Ci, N.ptr(wb), Co, N.ptr(pre),
                                          N.ptr(dact), N.ptr(dx), N.ptr(dw), N.ptr(db),
                                          N.ptr(ws), ws.numel(), N.stream_ptr(x.device)),
                "dm_conv3d_s2_backward")
        return (dx.to(x.dtype) if dx is not None else None), dw, db


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
    """Noisy normalised 64^3 images of ``verts[n, nv, 3]`` (one BatchRenderer launch set)."""
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
    return (noisy - lo) / (hi - lo)


def train_learned_init(n_train, epochs, batch=64, lr=1e-3, seed=0, device="cuda",
                       model=None, log=None):
    """Render ``n_train`` pairs with the package's renderer, then train with Adam on
    the vertex-position MSE.  Returns (model, sampler, per-epoch losses)."""
    rng = np.random.default_rng(seed)
    sampler = ShapeSampler()
    imgs, disps = [], []
    tmpl = torch.tensor(sampler.template, dtype=torch.float32, device=device)
    for s in range(0, n_train, batch):
        k = min(batch, n_train - s)
        v, sig = sampler.sample(k, rng)
        imgs.append(render_batch(v, sig, sampler.faces, rng.integers(1 << 30), device)
                    .to(torch.bfloat16))
        disps.append(torch.tensor(v, dtype=torch.float32, device=device) - tmpl)
    imgs = torch.cat(imgs)
    disps = torch.cat(disps)
    model = (model or LearnedInit(len(sampler.template), seed=seed)).to(device)
    opt = torch.optim.Adam(model.parameters(), lr=lr)
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
            tot += loss.detach() * len(idx)
        hist.append(float(tot) / n_train)
        if log:
            log(f"epoch {ep}: vertex MSE {hist[-1]:.3e}")
    return model, sampler, hist
