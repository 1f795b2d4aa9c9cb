"""numpy dtypes and ctypes structures for the C-ABI structs in include/tfg_pt.h.

Each layout is byte-compatible with the reference struct of the same name
(vector3d.h, color.h, primitiva.h, luzPuntual.h, camara.h, mlp_types.h,
tinybvh_wrapper.h); the sizes are asserted at import.
"""
from __future__ import annotations

import ctypes

import numpy as np

ESFERA, PLANO, TRIANGULO = 0, 1, 2

VEC3D = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8")])
COLOR = np.dtype([("r", "<f4"), ("g", "<f4"), ("b", "<f4")])

# Primitiva (primitiva.h:19-41): header + 144-byte union at offset 56.  The
# union is exposed as 18 doubles (`u`); sphere radius / plane distance are the
# float at byte 80 (`u_f32_80`), overlapping u[3].
PRIMITIVA = np.dtype({
    "names": ["tipo", "emision", "difuso", "especular", "transmision", "indice_refraccion", "u"],
    "formats": ["<i4", COLOR, COLOR, COLOR, COLOR, "<f4", ("<f8", 18)],
    "offsets": [0, 4, 16, 28, 40, 52, 56],
    "itemsize": 200,
})
LUZ = np.dtype({"names": ["posicion", "intensidad"], "formats": [VEC3D, COLOR], "offsets": [0, 24], "itemsize": 40})
CAMARA = np.dtype({
    "names": ["posicion", "frente", "arriba", "izquierda", "ancho_plano", "alto_plano", "distancia_focal"],
    "formats": [VEC3D, VEC3D, VEC3D, VEC3D, "<f4", "<f4", "<f4"],
    "offsets": [0, 24, 48, 72, 96, 100, 104],
    "itemsize": 112,
})
DATOS_MLP = np.dtype({
    "names": ["posicion", "direccion", "normal", "difuso", "especular", "color"],
    "formats": [VEC3D, VEC3D, VEC3D, COLOR, COLOR, COLOR],
    "offsets": [0, 24, 48, 72, 84, 96],
    "itemsize": 112,
})
GEO = np.dtype({
    "names": ["posicion", "direccion", "normal", "difuso", "especular"],
    "formats": [VEC3D, VEC3D, VEC3D, COLOR, COLOR],
    "offsets": [0, 24, 48, 72, 84],
    "itemsize": 96,
})
REGISTRO = np.dtype({
    "names": ["head", "tail", "luz_acumulada_sufijo", "throughput_sufijo", "factor_normalizacion", "valido"],
    "formats": [GEO, GEO, COLOR, COLOR, COLOR, "u1"],
    "offsets": [0, 96, 192, 204, 216, 228],
    "itemsize": 232,
})
BOUNDS = np.dtype({"names": ["min", "max"], "formats": [VEC3D, VEC3D], "offsets": [0, 24], "itemsize": 48})

assert PRIMITIVA.itemsize == 200 and LUZ.itemsize == 40 and CAMARA.itemsize == 112
assert DATOS_MLP.itemsize == 112 and REGISTRO.itemsize == 232 and BOUNDS.itemsize == 48


def set_sphere_radius(prims: np.ndarray, idx, r) -> None:
    """Store the float radius (or plane distance) at byte 80 of a Primitiva."""
    raw = prims.view(np.uint8).reshape(len(prims), 200)
    vals = np.asarray(r, dtype="<f4").reshape(-1)
    sel = np.arange(len(prims))[idx].reshape(-1)
    raw[sel, 80:84] = vals.view(np.uint8).reshape(-1, 4)


def get_f32_80(prims: np.ndarray) -> np.ndarray:
    raw = prims.view(np.uint8).reshape(len(prims), 200)
    return raw[:, 80:84].copy().view("<f4").reshape(-1)


class CTinyBVHD_GPU(ctypes.Structure):
    _fields_ = [("d_nodos", ctypes.c_void_p), ("d_tris", ctypes.c_void_p),
                ("num_nodos", ctypes.c_uint32), ("num_tris", ctypes.c_uint32)]


class CTinyBVH(ctypes.Structure):
    _fields_ = [("ref", CTinyBVHD_GPU), ("d_tris_wt", ctypes.c_void_p), ("d_primitivas", ctypes.c_void_p),
                ("num_primitivas", ctypes.c_uint32), ("max_depth", ctypes.c_uint32)]


class CCWBVHHost(ctypes.Structure):
    _fields_ = [("nodes", ctypes.POINTER(ctypes.c_float)), ("tris_ref", ctypes.POINTER(ctypes.c_float)),
                ("tris_wt", ctypes.POINTER(ctypes.c_float)), ("num_nodes", ctypes.c_uint32),
                ("num_tris", ctypes.c_uint32), ("max_depth", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class CRenderParams(ctypes.Structure):
    _fields_ = [("max_depth", ctypes.c_int32), ("rr_min_depth", ctypes.c_int32), ("shadow_mesh", ctypes.c_int32),
                ("tri_format", ctypes.c_int32), ("spp", ctypes.c_int32), ("accumulate", ctypes.c_int32),
                ("profile", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class CRenderProfile(ctypes.Structure):
    _fields_ = [("ms", ctypes.c_double * 5), ("launches", ctypes.c_uint64 * 5), ("rays", ctypes.c_uint64),
                ("nodes", ctypes.c_uint64), ("tri_tests", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64),
                ("shadow_nodes", ctypes.c_uint64), ("shadow_tri_tests", ctypes.c_uint64)]


class CHashGridConfig(ctypes.Structure):
    _fields_ = [("n_levels", ctypes.c_int32), ("log2_hashmap_size", ctypes.c_int32),
                ("base_resolution", ctypes.c_float), ("per_level_scale", ctypes.c_float),
                ("reserved", ctypes.c_int32 * 4)]


class CRenderScene(ctypes.Structure):
    _fields_ = [("camara", ctypes.c_void_p), ("primitivas", ctypes.c_void_p), ("num_primitivas", ctypes.c_int32),
                ("num_luces", ctypes.c_int32), ("luces", ctypes.c_void_p), ("ancho_img", ctypes.c_int32),
                ("alto_img", ctypes.c_int32), ("nodos_bvh", ctypes.c_void_p), ("tris_wt", ctypes.c_void_p),
                ("primitivas_bvh", ctypes.c_void_p), ("num_prims_bvh", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("imagen", ctypes.c_void_p), ("accum", ctypes.c_void_p)]


assert ctypes.sizeof(CRenderScene) == 88


class CRenderTuning(ctypes.Structure):
    _fields_ = [("wavefront_paths", ctypes.c_int32), ("trace_threads", ctypes.c_int32),
                ("trace_warps_per_sm", ctypes.c_int32), ("refill_min", ctypes.c_int32),
                ("shadow_one_lane", ctypes.c_int32), ("refill_min_primary", ctypes.c_int32),
                ("overlap_shadow", ctypes.c_int32), ("reserved", ctypes.c_int32 * 1)]


class CTuneRecord(ctypes.Structure):
    _fields_ = [("tuning", CRenderTuning), ("ms", ctypes.c_float), ("reserved", ctypes.c_int32)]


class CMlpTuning(ctypes.Structure):
    _fields_ = [("wgrad_tiles_per_cta", ctypes.c_int32), ("infer_ctas", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 2)]


assert ctypes.sizeof(CRenderTuning) == 32 and ctypes.sizeof(CTuneRecord) == 40 and ctypes.sizeof(CMlpTuning) == 16


class CImagenGPU(ctypes.Structure):
    _fields_ = [("anchura", ctypes.c_int32), ("altura", ctypes.c_int32), ("datos", ctypes.c_void_p)]


assert ctypes.sizeof(CTinyBVHD_GPU) == 24 and ctypes.sizeof(CImagenGPU) == 16


class CNrcFrameConfig(ctypes.Structure):
    _fields_ = [("train_steps", ctypes.c_int32), ("max_records", ctypes.c_uint32), ("min_records", ctypes.c_uint32),
                ("warmup", ctypes.c_int32), ("gate_threshold", ctypes.c_float), ("use_graph", ctypes.c_int32),
                ("footprint", ctypes.c_float), ("train_fraction", ctypes.c_float)]


class CNrcBuffers(ctypes.Structure):
    _fields_ = [("img", ctypes.c_void_p), ("accum", ctypes.c_void_p), ("infer", ctypes.c_void_p),
                ("thr", ctypes.c_void_p), ("regs", ctypes.c_void_p), ("counter", ctypes.c_void_p),
                ("ring_cap", ctypes.c_uint32), ("reserved", ctypes.c_uint32), ("tail_in", ctypes.c_void_p),
                ("tail_pred", ctypes.c_void_p), ("train_buf", ctypes.c_void_p)]


class CNrcSceneFrame(ctypes.Structure):
    """TfgNrcSceneFrame: one scene of tfgNrcFrameBatch (104 bytes)."""
    _fields_ = [("mlp", ctypes.c_void_p), ("cfg", ctypes.c_void_p), ("params", ctypes.c_void_p),
                ("camara", ctypes.c_void_p), ("primitivas", ctypes.c_void_p), ("luces", ctypes.c_void_p),
                ("bvh", ctypes.c_void_p), ("tris_wt", ctypes.c_void_p), ("primitivas_bvh", ctypes.c_void_p),
                ("buffers", ctypes.c_void_p), ("num_primitivas", ctypes.c_int32), ("num_luces", ctypes.c_int32),
                ("num_prims_bvh", ctypes.c_int32), ("ancho_img", ctypes.c_int32), ("alto_img", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


assert ctypes.sizeof(CNrcSceneFrame) == 104
