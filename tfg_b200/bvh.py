"""Host-side CWBVH build (tfgCWBVHBuild) returned as numpy arrays.

The same builder runs inside tfgTinyBVHConstruir, so for the same triangles
these arrays are exactly what the device holds.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .structs import CCWBVHHost, TRIANGULO


@dataclass
class HostBVH:
    nodes: np.ndarray      # float32 (num_nodes, 20)
    tris_ref: np.ndarray   # float32 (num_tris, 16)
    tris_wt: np.ndarray    # float32 (num_tris, 12)
    max_depth: int

    @property
    def num_nodes(self) -> int:
        return len(self.nodes)

    @property
    def num_tris(self) -> int:
        return len(self.tris_ref)


def triangle_vertices(mesh: np.ndarray) -> np.ndarray:
    """(n, 9) float32 vertices of the TRIANGULO entries, in input order
    (tinybvh_wrapper.cpp:36-44 keeps only triangles, in order)."""
    tri = mesh[mesh["tipo"] == TRIANGULO]
    return np.ascontiguousarray(tri["u"][:, :9].astype(np.float32))


def build_host(verts: np.ndarray) -> HostBVH:
    verts = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 9)
    h = CCWBVHHost()
    _lib.call("tfgCWBVHBuild", verts.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), len(verts), ctypes.byref(h))
    try:
        nodes = np.ctypeslib.as_array(h.nodes, shape=(h.num_nodes * 20,)).copy().reshape(-1, 20)
        tr = np.ctypeslib.as_array(h.tris_ref, shape=(h.num_tris * 16,)).copy().reshape(-1, 16)
        tw = np.ctypeslib.as_array(h.tris_wt, shape=(h.num_tris * 12,)).copy().reshape(-1, 12)
        return HostBVH(nodes, tr, tw, int(h.max_depth))
    finally:
        _lib.lib.tfgCWBVHFree(ctypes.byref(h))
