"""Shared test utilities."""
from __future__ import annotations

import ctypes

import numpy as np

from tfg_b200 import _lib
from tfg_b200.structs import CRenderParams


def rel_mse(x: np.ndarray, r: np.ndarray) -> float:
    """Mean over pixels and channels of (x - r)^2 / (r^2 + 1e-2), in FP64."""
    x = np.asarray(x, np.float64)
    r = np.asarray(r, np.float64)
    return float(np.mean((x - r) ** 2 / (r ** 2 + 1e-2)))


def reference_params(**over) -> CRenderParams:
    p = CRenderParams()
    _lib.lib.tfgRenderParamsReference(ctypes.byref(p))
    for k, v in over.items():
        setattr(p, k, v)
    return p


def oracle_image(orc, scene, hb, frame, prm=None, nthreads=8, use_inf=0, train=0, want_nrc=False):
    """CPU-oracle render of one sample; returns img (H, W, 3) [and NRC outputs]."""
    from tfg_b200.structs import DATOS_MLP, REGISTRO
    prm = prm or reference_params()
    W, H = scene.width, scene.height
    img = np.zeros((H, W, 3), np.float32)
    infer = thr = regs = flags = None
    if want_nrc:
        infer = np.zeros(W * H, DATOS_MLP)
        thr = np.zeros((W * H, 3), np.float32)
        regs = np.zeros(W * H, REGISTRO)
        flags = np.zeros(W * H, np.uint8)
    orc.cpu.orc_render(orc.p(scene.prims), len(scene.prims), orc.p(scene.lights), len(scene.lights),
                       orc.p(hb.nodes), orc.p(hb.tris_ref), orc.p(scene.mesh), len(scene.mesh), orc.p(scene.camera),
                       W, H, frame, ctypes.addressof(prm), 0, H, orc.p(img), orc.p(infer), orc.p(thr), orc.p(regs),
                       orc.p(flags), use_inf, train, nthreads)
    if want_nrc:
        return img, infer, thr, regs, flags
    return img


# ---------------------------------------------------------------- cache-network parity
# The cache kernels are checked against an FP64 model that applies their own
# roundings to their own layer-0 operands (tfgMlpEncodeFeatures): FP16 / BF16
# weights and hidden activations in inference; in training an FP16 forward
# pass, BF16 loss and layer-output gradients, BF16 backward weights and
# BF16-rounded layer inputs for the weight gradients.  What is left is the
# order of the FP32 sums, and an activation that lands on the other side of a
# rounding boundary than in the model.
# Measured on B200 (1000 queries, every width, depth and encoding): max
# 3.0e-3, mean 4e-5; gradients 1.9e-3 at most (7 hidden layers), loss 2e-6.
INFER_MAX = 5e-3      # largest |kernel - model| / mean |model output|
INFER_MEAN = 1e-4
GRAD_REL = 5e-3       # per layer: |g - model|_2 / |model|_2
LOSS_REL = 1e-4


def cache_inference_error(mlp, datos_dev, n, got, kind="f16"):
    """(max, mean) of |got - model| / mean|model| for inference of n queries."""
    import numpy as np

    from oracle import mlp_oracle as mo
    from tfg_b200.nrc import EMA, WEIGHTS, split_layers
    x = mlp.encode_features(datos_dev, n).cpu().numpy().astype(np.float64)
    st = mlp.state()
    if st["adam_t"] > 0:
        # inference reads the weight average debiased by 1 - decay^t, all in FP32
        debias = np.float32(1.0) - np.float32(0.99) ** np.float32(st["adam_t"])
        w = (mlp.get_params(EMA) / debias).astype(np.float32)
    else:
        w = mlp.get_params(WEIGHTS)
    raw = mo.forward_operands(split_layers(w), x, kind)
    want = mo.scrub(raw)
    scale = np.abs(raw).mean() + 1e-3
    err = np.abs(np.asarray(got, np.float64) - want) / scale
    return float(err.max()), float(err.mean())


def kchunk_columns(cols: int) -> list[int]:
    """Columns on either side of every 16-feature boundary of a K dimension
    (one tcgen05 MMA of 16-bit operands covers 16 features)."""
    out = []
    for b in range(16, cols, 16):
        out += [b - 1, b]
    return out


def check_cache_gradients(mlp, sel_dev, y, g, loss, bias_col: int, g_table=None, corners=None,
                          table_cols: int = 0, tol_rel=GRAD_REL):
    """Layer gradients (and the hash-grid table gradient) of one training
    batch against the operand model; `sel_dev` holds the batch's samples in
    the order the kernel drew them.  Element-wise on the bias column of layer
    0 and on every K-chunk boundary column: |g - model| <= 0.05 |model| +
    0.01 rms(layer)."""
    import numpy as np

    from oracle import mlp_oracle as mo
    from tfg_b200.nrc import WEIGHTS, split_layers
    n = len(y)
    x = mlp.encode_features(sel_dev, n, training=True).cpu().numpy().astype(np.float64)
    W = split_layers(mlp.get_params(WEIGHTS))
    ref_loss, ref, dx = mo.loss_and_grad_operands(W, x, y)
    assert abs(loss - ref_loss) / ref_loss < LOSS_REL, (loss, ref_loss)
    report = []
    for l, (gg, rr) in enumerate(zip(split_layers(g), ref)):
        rel = float(np.linalg.norm(gg - rr) / (np.linalg.norm(rr) + 1e-30))
        report.append(rel)
        assert rel < tol_rel, f"layer {l}: relative gradient error {rel:.3e} (all: {report})"
        rms = float(np.sqrt(np.mean(rr ** 2)))
        cols = kchunk_columns(rr.shape[1]) + ([bias_col] if l == 0 else [])
        d = np.abs(gg[:, cols] - rr[:, cols])
        bound = 0.05 * np.abs(rr[:, cols]) + 0.01 * rms
        assert (d <= bound).all(), f"layer {l}: column check, worst {float((d - bound).max()):.3e} over rms {rms:.3e}"
    if g_table is not None:
        ref_t = mo.table_grad(dx[:, :table_cols], corners, len(g_table))
        rel = float(np.linalg.norm(g_table - ref_t) / np.linalg.norm(ref_t))
        report.append(rel)
        assert rel < tol_rel, f"table gradient: relative error {rel:.3e}"
        assert (g_table[ref_t == 0] == 0).all()
    return report
