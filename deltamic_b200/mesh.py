"""Synthetic surface meshes: icospheres and spherical-harmonic shapes.

The reference draws its meshes from trimesh (``trimesh.primitives.Sphere``,
``Examples/Gradient_Descent.ipynb`` cell 2) and from ``.obj`` files.  trimesh is
not a dependency here; this module builds the same family of shapes itself:

* ``icosphere(level, radius)`` -- a regular icosahedron subdivided ``level``
  times (each triangle split in four, new vertices pushed to the sphere), so
  level L has ``10*4**L + 2`` vertices and ``20*4**L`` faces (level 3: 642 / 1,280,
  level 5: 10,242 / 20,480).  Faces are oriented outward.
* ``sh_perturb(verts, lmax, amp, rng)`` -- radial perturbation
  ``r = r0 * (1 + sum_{l=1..lmax} sum_m a_lm Y_lm)`` with real spherical harmonics
  and ``a_lm ~ N(0, (amp/l)^2)``.

Everything is plain numpy (float64) so that the same inputs can be handed to the
CUDA path and to the CPU oracle.
"""
from __future__ import annotations

import math

import numpy as np

__all__ = ["icosphere", "real_sph_harm", "sh_radial_field", "sh_perturb",
           "jitter", "random_sh_shape"]


def _icosahedron():
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([
        [-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
        [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
        [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1],
    ], dtype=np.float64)
    f = np.array([
        [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
        [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
        [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
        [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1],
    ], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v, f


def icosphere(level: int, radius: float = 1.0, center=(0.0, 0.0, 0.0)):
    """Return ``(verts[nv,3] float64, faces[nt,3] int64)`` of a subdivided icosahedron."""
    if level < 0:
        raise ValueError("level must be >= 0")
    v, f = _icosahedron()
    verts = [row for row in v]
    for _ in range(level):
        cache: dict[tuple[int, int], int] = {}

        def midpoint(i: int, j: int) -> int:
            key = (i, j) if i < j else (j, i)
            idx = cache.get(key)
            if idx is None:
                m = verts[i] + verts[j]
                m = m / np.linalg.norm(m)
                idx = len(verts)
                verts.append(m)
                cache[key] = idx
            return idx

        nf = np.empty((4 * len(f), 3), dtype=np.int64)
        for k, (a, b, c) in enumerate(f):
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf[4 * k + 0] = (a, ab, ca)
            nf[4 * k + 1] = (b, bc, ab)
            nf[4 * k + 2] = (c, ca, bc)
            nf[4 * k + 3] = (ab, bc, ca)
        f = nf
    out = np.asarray(verts, dtype=np.float64) * float(radius)
    out += np.asarray(center, dtype=np.float64)
    return out, f


def real_sph_harm(l: int, m: int, theta: np.ndarray, phi: np.ndarray) -> np.ndarray:
    """Orthonormal real spherical harmonic Y_lm(theta=polar, phi=azimuth).

    Associated Legendre functions are evaluated by the standard upward
    recurrence in ``l`` (no Condon-Shortley phase), then combined with
    ``cos(m phi)`` / ``sin(|m| phi)``.
    """
    am = abs(m)
    x = np.cos(theta)
    s = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    # P_m^m
    pmm = np.ones_like(x)
    for k in range(1, am + 1):
        pmm = pmm * (2 * k - 1) * s
    if l == am:
        plm = pmm
    else:
        pm1 = x * (2 * am + 1) * pmm
        if l == am + 1:
            plm = pm1
        else:
            p_prev, p_cur = pmm, pm1
            for ll in range(am + 2, l + 1):
                p_next = ((2 * ll - 1) * x * p_cur - (ll + am - 1) * p_prev) / (ll - am)
                p_prev, p_cur = p_cur, p_next
            plm = p_cur
    norm = math.sqrt((2 * l + 1) / (4 * math.pi)
                     * math.factorial(l - am) / math.factorial(l + am))
    if m == 0:
        return norm * plm
    if m > 0:
        return math.sqrt(2.0) * norm * plm * np.cos(am * phi)
    return math.sqrt(2.0) * norm * plm * np.sin(am * phi)


def sh_radial_field(dirs: np.ndarray, coeffs: dict) -> np.ndarray:
    """sum_{(l,m)} a_lm Y_lm(direction) for unit vectors ``dirs[n,3]``."""
    theta = np.arccos(np.clip(dirs[:, 2], -1.0, 1.0))
    phi = np.arctan2(dirs[:, 1], dirs[:, 0])
    out = np.zeros(len(dirs))
    for (l, m), a in coeffs.items():
        out += a * real_sph_harm(l, m, theta, phi)
    return out


def sh_perturb(verts: np.ndarray, lmax: int, amp: float, rng: np.random.Generator,
               radius: float | None = None, center=(0.0, 0.0, 0.0)):
    """Radially perturb a (centred) sphere mesh: ``r = r0 (1 + sum a_lm Y_lm)``.

    ``a_lm ~ N(0, (amp / l)^2)`` for ``l = 1..lmax`` and ``m = -l..l``, drawn from
    ``rng`` in a fixed order.  Returns ``(new_verts, coeffs)``.
    """
    c = np.asarray(center, dtype=np.float64)
    d = verts - c
    r0 = np.linalg.norm(d, axis=1)
    if radius is None:
        radius = float(np.mean(r0))
    dirs = d / r0[:, None]
    coeffs = {}
    for l in range(1, lmax + 1):
        for m in range(-l, l + 1):
            coeffs[(l, m)] = rng.normal(0.0, amp / l)
    r = radius * (1.0 + sh_radial_field(dirs, coeffs))
    return c + dirs * r[:, None], coeffs


def jitter(verts: np.ndarray, std: float, rng: np.random.Generator) -> np.ndarray:
    return verts + rng.normal(0.0, std, size=verts.shape)


def random_sh_shape(level: int, radius: float, lmax: int, amp: float, seed: int):
    """Icosphere of ``level`` with an SH radial perturbation drawn from ``seed``."""
    rng = np.random.default_rng(seed)
    v, f = icosphere(level, radius)
    v, _ = sh_perturb(v, lmax, amp, rng, radius=radius)
    return v, f
