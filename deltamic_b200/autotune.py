"""Autotuner for the meshFT kernels' tile shapes.

The library compiles several tile-shape variants of the forward kernel
(frequencies per thread x threads per CTA x waves) and of the adjoint kernel
(faces per thread x threads per CTA x waves).  ``tune`` times every variant on
the caller's own problem and keeps the fastest per *size class* (log2 of the face
count, log2 of the band size); the choice is remembered for the process and, if
``$DM_AUTOTUNE_CACHE`` names a JSON file, across processes.
"""
from __future__ import annotations

import ctypes
import json
import math
import os

import torch

from . import _native as N
from . import ops

__all__ = ["size_class", "tune", "apply", "current"]

_CACHE: dict = {}


def size_class(nt: int, nband: int) -> str:
    return f"{int(math.log2(max(nt, 1)))}:{int(math.log2(max(nband, 1)))}"


def _load():
    path = os.environ.get("DM_AUTOTUNE_CACHE")
    if path and os.path.exists(path):
        try:
            with open(path) as f:
                _CACHE.update({k: tuple(v) for k, v in json.load(f).items()})
        except (OSError, ValueError):
            pass


def _save():
    path = os.environ.get("DM_AUTOTUNE_CACHE")
    if path:
        try:
            with open(path, "w") as f:
                json.dump(_CACHE, f)
        except OSError:
            pass


def current():
    f, b, nf, nb = (N._INT() for _ in range(4))
    N.lib().dm_get_variants(ctypes.byref(f), ctypes.byref(b), ctypes.byref(nf), ctypes.byref(nb))
    return f.value, b.value, nf.value, nb.value


def apply(variants) -> None:
    N.check(N.lib().dm_set_variants(int(variants[0]), int(variants[1])), "dm_set_variants")


def _time(fn, reps, trials=3):
    """Fastest of ``trials`` event-timed runs of ``reps`` calls each (after one
    untimed call): variants a few percent apart are told apart reliably."""
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(trials):
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / reps)
    return best


def _pick(n_variants, set_variant, fn, reps, trials=4):
    """Index of the fastest variant: every trial times each variant once, in
    turn, so clock changes during tuning fall on all variants alike; a variant
    keeps its fastest trial."""
    best = [float("inf")] * n_variants
    for v in range(n_variants):  # warm-up: first launch of each variant
        set_variant(v)
        fn()
    for _ in range(trials):
        for v in range(n_variants):
            set_variant(v)
            best[v] = min(best[v], _time(fn, reps, trials=1))
    return min(range(n_variants), key=lambda v: best[v])


def tune(verts, faces, coeff, grid, band, reps=4, force=False):
    """Pick and apply the fastest (forward, adjoint) variants for this size class."""
    if not _CACHE:
        _load()
    key = size_class(int(faces.shape[0]), int(band.numel()))
    if key in _CACHE and not force:
        apply(_CACHE[key])
        return _CACHE[key]
    f0, b0, nf, nb = current()
    g = torch.ones(band.numel(), dtype=torch.complex64, device=verts.device)
    ft = ops.meshft_list(verts, faces, coeff, grid, band)
    best_f = _pick(nf, lambda v: apply((v, b0)),
                   lambda: ops.meshft_list(verts, faces, coeff, grid, band), reps)
    best_b = _pick(nb, lambda v: apply((best_f, v)),
                   lambda: ops.meshft_backward_list(verts, faces, coeff, grid, band, ft,
                                                    grad_list=g, want_coeff=False), reps)
    _CACHE[key] = (best_f, best_b)
    apply(_CACHE[key])
    _save()
    return _CACHE[key]
