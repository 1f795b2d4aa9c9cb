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

def shapes(hidden_layers: int = 5) -> list[tuple[int, int]]:
    return [(64, 96)] + [(64, 64)] * (hidden_layers - 1) + [(16, 64)]


SHAPES = shapes(5)


def split(flat):
    """Layer matrices of a flat parameter array; its length gives the depth."""
    hidden = (len(flat) - 6144 - 1024) // 4096 + 1
    out, o = [], 0
    for r, c in shapes(hidden):
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


def round_bf16(a) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even) and back to FP64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _e4m3_grid() -> np.ndarray:
    """Every finite non-negative E4M3 value (bias 7, 3 mantissa bits, max 448)."""
    vals = [m / 8.0 * 2.0 ** -6 for m in range(8)]                        # subnormals
    vals += [(1.0 + m / 8.0) * 2.0 ** (e - 7) for e in range(1, 16) for m in range(8)
             if not (e == 15 and m == 7)]                                  # S.1111.111 is NaN
    return np.array(sorted(set(vals)))


_E4M3 = _e4m3_grid()


def round_e4m3(a) -> np.ndarray:
    """Round to the nearest E4M3 value, ties to even mantissa, saturating at
    +-448 (the satfinite conversion)."""
    x = np.asarray(a, np.float64)
    s, m = np.sign(x), np.minimum(np.abs(x), 448.0)
    i = np.clip(np.searchsorted(_E4M3, m), 1, len(_E4M3) - 1)
    lo, hi = _E4M3[i - 1], _E4M3[i]
    pick_hi = (m - lo > hi - m) | ((m - lo == hi - m) & ((i % 2) == 0))   # grid index parity = mantissa parity
    r = np.where(pick_hi, hi, lo)
    r = np.where(m >= _E4M3[-1], _E4M3[-1], r)
    return s * r


def forward_quantized(W, x, kind: str, amax=None):
    """Output (first 3 columns) of the network with operands rounded as the
    BF16 or FP8 inference kernels round them: BF16 rounds weights and every
    layer input; FP8 scales layer l's input by q = 448 / (2 amax[l]) and its
    weights by wq = 448 / max|W_l|, rounds both to E4M3 and rescales the
    FP64 product by 1 / (q wq)."""
    h = x
    for l, w in enumerate(W):
        if kind == "bf16":
            z = round_bf16(h) @ round_bf16(w).T
        else:
            q = 448.0 / (2.0 * amax[l])
            wq = 448.0 / np.abs(w).max()
            z = (round_e4m3(h * q) @ round_e4m3(w * wq).T) / (q * wq)
        h = np.maximum(z, 0.0) if l < len(W) - 1 else z
    return h[:, :3]


def layer_input_amax(W, x) -> list[float]:
    """Largest |input| of each layer (the encoded features' amax is at least 1)."""
    _, hs, _ = forward(W, x)
    out = [max(1.0, float(np.abs(x[:, 72:85]).max()))]
    out += [float(np.abs(h).max()) for h in hs[1:len(W)]]
    return out
