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
