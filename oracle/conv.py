"""Oracle: 3x3x3 stride-2 padding-1 convolution + GELU and its adjoint (numpy
float64, channels-last) -- TEST INFRASTRUCTURE ONLY.

Layout as the CUDA kernels: x[B,D,H,W,Ci], w[K,Co] with row k = ((kd*3+kh)*3+kw)*Ci
+ ci (K = 27*Ci; extra padding rows of the device layout are ignored), bias[Co];
output (D+1)/2 x (H+1)/2 x (W+1)/2 voxels.
"""
from __future__ import annotations

import math

import numpy as np


def _gelu(x):
    erf = np.vectorize(math.erf)
    return 0.5 * x * (1.0 + erf(x / math.sqrt(2.0)))


def _gelu_grad(x):
    erf = np.vectorize(math.erf)
    return 0.5 * (1.0 + erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2 * math.pi)


def im2col(x):
    B, D, H, W, Ci = x.shape
    Do, Ho, Wo = (D + 1) // 2, (H + 1) // 2, (W + 1) // 2
    xp = np.zeros((B, D + 2, H + 2, W + 2, Ci))
    xp[:, 1:D + 1, 1:H + 1, 1:W + 1] = x
    cols = np.empty((B, Do, Ho, Wo, 27, Ci))
    for kd in range(3):
        for kh in range(3):
            for kw in range(3):
                cols[:, :, :, :, (kd * 3 + kh) * 3 + kw] = xp[:, kd:kd + 2 * Do:2,
                                                                 kh:kh + 2 * Ho:2,
                                                                 kw:kw + 2 * Wo:2]
    return cols.reshape(B * Do * Ho * Wo, 27 * Ci), (Do, Ho, Wo)


def conv_forward(x, w, b):
    """Returns (pre, act) with shape [B, Do, Ho, Wo, Co]."""
    x = np.asarray(x, np.float64)
    B = x.shape[0]
    A, (Do, Ho, Wo) = im2col(x)
    K = A.shape[1]
    pre = A @ np.asarray(w, np.float64)[:K] + np.asarray(b, np.float64)
    pre = pre.reshape(B, Do, Ho, Wo, -1)
    return pre, _gelu(pre)


def conv_backward(x, w, pre, dact):
    """Returns (dx, dw[K,Co], db[Co]) for dL/dact = ``dact``."""
    x = np.asarray(x, np.float64)
    B, D, H, W, Ci = x.shape
    A, (Do, Ho, Wo) = im2col(x)
    K = A.shape[1]
    dp = (np.asarray(dact, np.float64) * _gelu_grad(np.asarray(pre, np.float64)))
    dp2 = dp.reshape(-1, dp.shape[-1])
    dw = A.T @ dp2
    db = dp2.sum(axis=0)
    dcols = (dp2 @ np.asarray(w, np.float64)[:K].T).reshape(B, Do, Ho, Wo, 27, Ci)
    dxp = np.zeros((B, D + 2, H + 2, W + 2, Ci))
    for kd in range(3):
        for kh in range(3):
            for kw in range(3):
                dxp[:, kd:kd + 2 * Do:2, kh:kh + 2 * Ho:2, kw:kw + 2 * Wo:2] += \
                    dcols[:, :, :, :, (kd * 3 + kh) * 3 + kw]
    return dxp[:, 1:D + 1, 1:H + 1, 1:W + 1], dw, db
