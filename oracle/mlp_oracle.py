"""FP64 numpy model of the cache MLP -- TEST INFRASTRUCTURE ONLY.

The forward pass, the relative-L2-luminance loss and its gradient, Adam and
the weight EMA, written from their definitions (Mueller et al. 2021, "Real-
time Neural Radiance Caching for Path Tracing"; Kingma & Ba 2015) for the
network the product kernels implement: 12-band frequency encoding of the
normalised position + 12 raw inputs + constant 1 -> 5 x 64 ReLU -> 3.
Input rows follow the reference's 15-float layout (NrcKernel.cu:18-97).

The reference's own input (mlp.cpp:22-49: tiny-cuda-nn's Composite of
HashGrid, OneBlob and Identity; tiny-cuda-nn is not in the reference tree
and its version is not pinned) is restated from the published methods: the
multiresolution hash encoding of Mueller, Evans, Schied and Keller 2022
("Instant Neural Graphics Primitives", Sec. 3: N_l = floor(N_min b^l),
trilinear interpolation of the 2^d corner features, the spatial hash
x * 1 ^ y * 2654435761 ^ z * 805459861 mod T, dense indexing where the
level's corners fit in T) and the one-blob encoding of Mueller et al. 2019
("Neural Importance Sampling", Sec. 4.3: k bins, a Gaussian of sigma 1/k
centred on the input, integrated over each bin).
"""
from __future__ import annotations

import numpy as np
from scipy.special import ndtr

def shapes(hidden_layers: int = 5, width: int = 64) -> list[tuple[int, int]]:
    return [(width, 96)] + [(width, width)] * (hidden_layers - 1) + [(16, width)]


SHAPES = shapes(5)


def split(flat):
    """Layer matrices of a flat parameter array; its length gives the depth
    and the width (64 or 128)."""
    for width in (64, 128):
        hidden = (len(flat) - 112 * width) // (width * width) + 1
        if hidden >= 1 and sum(r * c for r, c in shapes(hidden, width)) == len(flat):
            break
    out, o = [], 0
    for r, c in shapes(hidden, width):
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


def loss_and_grad(W, x, y, want_dx: bool = False):
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
    if want_dx:
        return loss, grads, dz @ W[0]     # gradient of the layer-0 input features
    return loss, grads


# ---------------------------------------------------------------- composite encoding
def hashgrid_levels(cfg: dict):
    """(N_l, dense) per level and the entries per level T."""
    T = 2 ** int(cfg["log2_hashmap_size"])
    out = []
    for l in range(int(cfg["n_levels"])):
        N = int(np.floor(float(np.float32(cfg["base_resolution"])) * float(np.float32(cfg["per_level_scale"])) ** l))
        out.append((N, (N + 1) ** 3 <= T))
    return out, T


def hash_index(x, y, z, N: int, dense: bool, T: int):
    x, y, z = (np.asarray(a, np.uint64) for a in (x, y, z))
    if dense:
        return x + np.uint64(N + 1) * (y + np.uint64(N + 1) * z)
    m = np.uint64(0xFFFFFFFF)
    return (x ^ ((y * np.uint64(2654435761)) & m) ^ ((z * np.uint64(805459861)) & m)) & np.uint64(T - 1)


def one_blob(s: np.ndarray, k: int = 4) -> np.ndarray:
    """One-blob bins (Mueller et al. 2019) of inputs s in [0, 1]: bin b holds
    the mass of a Gaussian of sigma 1/k centred at s that falls in
    [b/k, (b+1)/k), in FP64 (n x k)."""
    s = np.asarray(s, np.float64)
    cdf = [ndtr((b / k - s) * k) for b in range(k + 1)]
    return np.stack([cdf[b + 1] - cdf[b] for b in range(k)], 1)


def composite_encode(r15: np.ndarray, table: np.ndarray, cfg: dict):
    """Layer-0 input (n x 96) of the composite encoding -- 2L hash-grid
    features, 6 x 4 one-blob bins, 6 albedos, the constant 1 -- and, per
    level, the (flat table entry, trilinear weight) of the 8 corners of every
    sample's cell, for the table gradient.  The cell arithmetic is FP32, as in
    the kernels, so both pick the same cells."""
    levels, T = hashgrid_levels(cfg)
    n = len(r15)
    x = np.zeros((n, 96))
    tab = np.asarray(table, np.float64).reshape(len(levels), T, 2)
    p32 = r15[:, 0:3].astype(np.float32)
    corners = []
    for l, (N, dense) in enumerate(levels):
        pos = p32 * np.float32(N)
        c = np.minimum(np.floor(pos), np.float32(N - 1))
        i = c.astype(np.uint64)
        f = (pos - c).astype(np.float64)
        lst = []
        for k in range(8):
            ox, oy, oz = k & 1, (k >> 1) & 1, k >> 2
            q = hash_index(i[:, 0] + ox, i[:, 1] + oy, i[:, 2] + oz, N, dense, T).astype(np.int64)
            w = (f[:, 0] if ox else 1 - f[:, 0]) * (f[:, 1] if oy else 1 - f[:, 1]) * (f[:, 2] if oz else 1 - f[:, 2])
            x[:, 2 * l:2 * l + 2] += w[:, None] * tab[l, q]
            lst.append((l * T + q, w))
        corners.append(lst)
    for j in range(6):
        x[:, 32 + 4 * j:36 + 4 * j] = one_blob(r15[:, 3 + j])
    x[:, 56:62] = r15[:, 9:15]
    x[:, 62] = 1.0
    return x, corners


def table_grad(dx: np.ndarray, corners, size: int) -> np.ndarray:
    """Gradient of the flat [level][entry][feature] table from the gradient
    of the hash-grid features (dx[:, 2l], dx[:, 2l + 1] of level l)."""
    g = np.zeros(size)
    for l, lst in enumerate(corners):
        for q, w in lst:
            np.add.at(g, 2 * q, w * dx[:, 2 * l])
            np.add.at(g, 2 * q + 1, w * dx[:, 2 * l + 1])
    return g


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


def round_f16(a) -> np.ndarray:
    """Round to the nearest FP16 value (ties to even) and back to FP64; the
    value is first rounded to FP32, the kernels' accumulator type."""
    return np.asarray(a, np.float64).astype(np.float32).astype(np.float16).astype(np.float64)


def forward_operands(W, x, kind: str = "f16"):
    """Output (first 3 columns) of the network as the FP16 / BF16 inference
    kernels compute it from their own layer-0 operands `x` (the features
    tfgMlpEncodeFeatures returns, already rounded): weights rounded to the
    operand type, every hidden layer's ReLU output rounded to it before the
    next GEMM, products summed in FP64 (the kernels accumulate in FP32)."""
    rnd = round_f16 if kind == "f16" else round_bf16
    h = np.asarray(x, np.float64)
    for l, w in enumerate(W):
        z = h @ rnd(w).T
        if l < len(W) - 1:
            h = rnd(np.maximum(z, 0.0))
    return z[:, :3]


def loss_and_grad_operands(W, x, y):
    """Loss, layer gradients and the gradient of the layer-0 operands as the
    training kernels compute them from their own FP16 layer-0 operands `x`:
    FP16 forward pass (FP16 weights, every hidden ReLU output rounded to FP16
    for the next GEMM); the loss gradient and every layer-output gradient
    rounded to BF16; the backward GEMMs with BF16 weights; the weight
    gradients from the BF16-rounded layer inputs (the ReLU outputs rounded
    from their FP32 values) and output gradients; the layer-0 operand
    gradient (for the hash-grid tables) with FP16 layer-0 weights.  Sums in
    FP64."""
    W16 = [round_f16(w) for w in W]
    Wbf = [round_bf16(w) for w in W]
    L = len(W)
    h = np.asarray(x, np.float64)
    h_bf = [round_bf16(h)]
    zs = []
    for l in range(L):
        z = h @ W16[l].T
        zs.append(z)
        if l < L - 1:
            a = np.maximum(z, 0.0)
            h = round_f16(a)
            h_bf.append(round_bf16(a))
    pred = zs[-1][:, :3]
    lum = 0.299 * pred[:, 0] + 0.587 * pred[:, 1] + 0.114 * pred[:, 2]
    den = lum * lum + 0.01
    n = len(x)
    loss = float(np.sum((pred - y) ** 2 / den[:, None]) / (3 * n))
    g = np.zeros_like(zs[-1])
    g[:, :3] = 2.0 * (pred - y) / den[:, None]
    dz = round_bf16(g)
    grads = [None] * L
    for l in range(L - 1, -1, -1):
        grads[l] = dz.T @ h_bf[l] / (3 * n)
        if l > 0:
            dz = round_bf16((dz @ Wbf[l]) * (zs[l - 1] > 0))
    dx = dz @ W16[0] / (3 * n)
    return loss, grads, dx


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
