"""ctypes access to the oracles -- TEST INFRASTRUCTURE ONLY.

``cpu`` binds oracle/liboracle.so (the CPU restatement of the reference);
``ref`` binds oracle/_ref/libtfgref.so (the reference's own kernels built
for sm_100a), or is None when that file is absent.  Only tests/, the smoke
check and bench.py's CPU-baseline / reference legs use this module.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_float, c_int, c_uint32, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _load_cpu():
    from . import build_oracle
    build_oracle.build_cpu()
    lib = ctypes.CDLL(str(build_oracle.ORACLE_LIB))
    lib.orc_seed.restype = c_uint32
    lib.orc_seed.argtypes = [c_int, c_int, c_int]
    lib.orc_pcg_stream.argtypes = [c_uint32, c_int, c_void_p, c_void_p]
    lib.orc_trace_batch.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int]
    lib.orc_brute_batch.argtypes = [c_void_p, c_uint32, c_void_p, c_int, c_void_p, c_int]
    lib.orc_camera_rays.argtypes = [c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p]
    lib.orc_render.argtypes = [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_int, c_void_p,
                               c_int, c_int, c_int, c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p,
                               c_void_p, c_void_p, c_int, c_int, c_int]
    lib.orc_indices.argtypes = [c_void_p, c_int, c_int, c_uint32]
    lib.orc_train_rows.argtypes = [c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]
    lib.orc_infer_rows.argtypes = [c_void_p, c_int, c_int, c_void_p, c_void_p]
    lib.orc_scrub.argtypes = [c_void_p, c_void_p, c_int]
    lib.orc_composite.argtypes = [c_void_p, c_void_p, c_void_p, c_int]
    lib.orc_tonemap_filmic.argtypes = [c_void_p, c_int, c_int, c_void_p, c_void_p]
    lib.orc_targets.argtypes = [c_void_p, c_void_p, c_void_p, c_int]
    lib.orc_tail.argtypes = [c_void_p, c_void_p, c_int]
    lib.orc_default_camera.argtypes = [c_void_p, c_int, c_int]
    return lib


def _load_ref():
    from . import build_oracle
    try:
        path = build_oracle.build_ref()
    except RuntimeError:
        path = build_oracle.REF_LIB if build_oracle.REF_LIB.exists() else None
    if path is None or not Path(path).exists():
        return None
    lib = ctypes.CDLL(str(path))
    lib.ref_trace.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p]
    lib.ref_render_tiny.argtypes = [c_void_p, c_void_p, c_int, c_void_p, c_int, c_int, c_int, c_int, c_void_p,
                                    c_void_p, c_uint32, c_uint32, c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                                    c_int, c_void_p, c_void_p, c_int, c_int]
    lib.ref_camera.argtypes = [c_void_p, c_int, c_int]
    lib.ref_composite.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_int]
    lib.ref_targets.argtypes = [c_void_p, c_void_p, c_void_p, c_int]
    lib.ref_tail.argtypes = [c_void_p, c_void_p, c_int]
    lib.ref_indices.argtypes = [c_void_p, c_int, c_int, c_uint32]
    lib.ref_train_rows.argtypes = [c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]
    lib.ref_infer_rows.argtypes = [c_void_p, c_uint32, c_uint32, c_void_p, c_void_p]
    lib.ref_scrub.argtypes = [c_void_p, c_void_p, c_int]
    return lib


cpu = _load_cpu()
_ref = None
_ref_loaded = False


def ref():
    global _ref, _ref_loaded
    if not _ref_loaded:
        _ref = _load_ref()
        _ref_loaded = True
    return _ref


def p(a: np.ndarray) -> int | None:
    return None if a is None else a.ctypes.data


def pcg_stream(state: int, n: int) -> tuple[np.ndarray, np.ndarray]:
    u = np.zeros(n, np.uint32)
    f = np.zeros(n, np.float32)
    cpu.orc_pcg_stream(state, n, p(u), p(f))
    return u, f


def trace_batch(nodes: np.ndarray, tris_ref: np.ndarray, rays: np.ndarray, nthreads: int = 8):
    n = len(rays)
    hits = np.zeros((n, 4), np.float32)
    counts = np.zeros((n, 3), np.uint32)
    cpu.orc_trace_batch(p(nodes), p(tris_ref), p(rays), n, p(hits), p(counts), nthreads)
    return hits, counts


def brute_batch(tris_ref: np.ndarray, rays: np.ndarray, nthreads: int = 8):
    n = len(rays)
    hits = np.zeros((n, 4), np.float32)
    cpu.orc_brute_batch(p(tris_ref), len(tris_ref), p(rays), n, p(hits), nthreads)
    return hits


def camera_rays(cam: np.ndarray, W: int, H: int, frame: int, y0: int = 0, y1: int | None = None) -> np.ndarray:
    y1 = H if y1 is None else y1
    rays = np.zeros(((y1 - y0) * W, 8), np.float32)
    cpu.orc_camera_rays(p(cam), W, H, frame, y0, y1, p(rays))
    return rays
