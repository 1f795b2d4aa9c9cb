"""FP64 numpy model of the cache MLP -- TEST INFRASTRUCTURE ONLY.

The forward pass, the relative-L2-luminance loss and its gradient, Adam and
the weight EMA, written from their definitions (Mueller et al. 2021, "Real-
time Neural Radiance Caching for Path Tracing"; Kingma & Ba 2015) for the
network the product kernels implement: 12-band frequency encoding of the
normalised position + 12 raw inputs + constant 1 -> 5 x 64 ReLU -> 3.
Input rows follow the reference's 15-float layout (NrcKernel.cu:18-97).
"""
from __future__ import annotations

import numpy as np

SHAPES = [(64, 96), (64, 64), (64, 64), (64, 64), (64, 64), (16, 64)]


def split(flat):
    out, o = [], 0
    for r, c in SHAPES:
        out.append(np.asarray(flat[o:o + r * c], np.float64).reshape(r, c))
        o += r * c
    return out


def rows15(datos: np.ndarray, lo, hi) -> np.ndarray:
    """The reference's 15-float input row (NrcKernel.cu:18-47), float32 math."""
    n = len(datos)
    r = np.zeros((n, 15), np.float32)
    for j, k in enumerate("xyz"):
        v = datos["posicion"][k].astype(np.float32)
        a, b = np.float32(lo[j]), np.float32(hi[j])
        r[:, j] = np.clip((v - a) / (b - a), np.float32(0), np.float32(1))
        r[:, 3 + j] = datos["direccion"][k].astype(np.float32)
        r[:, 6 + j] = datos["normal"][k].astype(np.float32)
    for j, k in enumerate("rgb"):
        r[:, 9 + j] = datos["difuso"][k]
        r[:, 12 + j] = datos["especular"][k]
    return r


def encode(r15: np.ndarray) -> np.ndarray:
    n = len(r15)
    x = np.zeros((n, 96))
    p = r15[:, 0:3].astype(np.float64)
    for j in range(3):
        for b in range(12):
            a = (2.0 ** b) * np.pi * p[:, j]
            x[:, 24 * j + 2 * b] = np.sin(a)
            x[:, 24 * j + 2 * b + 1] = np.cos(a)
    x[:, 72:84] = r15[:, 3:15]
    x[:, 84] = 1.0
    return x


def forward(W, x):
    hs, zs = [x], []
    h = x
    for l, w in enumerate(W):
        z = h @ w.T
        zs.append(z)
        h = np.maximum(z, 0.0) if l < len(W) - 1 else z
        hs.append(h)
    return zs[-1][:, :3], hs, zs


def loss_and_grad(W, x, y):
    pred, hs, zs = forward(W, x)
    lum = 0.299 * pred[:, 0] + 0.587 * pred[:, 1] + 0.114 * pred[:, 2]
    den = lum * lum + 0.01
    n = len(x)
    loss = float(np.sum((pred - y) ** 2 / den[:, None]) / (3 * n))
    dz = np.zeros_like(zs[-1])
    dz[:, :3] = 2.0 * (pred - y) / den[:, None] / (3 * n)
    grads = [None] * len(W)
    for l in range(len(W) - 1, -1, -1):
        grads[l] = dz.T @ hs[l]
        if l > 0:
            dh = dz @ W[l]
            dz = dh * (zs[l - 1] > 0)
    return loss, grads


def scrub(c):
    c = np.where(c < 0, 0, c)
    c = np.where(np.isnan(c), 0, c)
    return np.minimum(c, 1e5)
