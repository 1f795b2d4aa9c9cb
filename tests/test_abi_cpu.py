"""C ABI checks that need no GPU: the library loads, exports every function
declared in include/tfg_pt.h, struct layouts match the reference's sizes, and
entry points reject bad arguments before touching the device."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def _declared_functions():
    text = (ROOT / "include" / "tfg_pt.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(tfg\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol(built):
    from tfg_b200 import _lib
    names = _declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(_lib.lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    # every declared function has a ctypes prototype in the binding
    assert set(names) <= set(_lib.exported_symbols())


def test_struct_sizes_match_reference():
    from tfg_b200 import structs as S
    assert S.PRIMITIVA.itemsize == 200          # measured on the reference with nvcc
    assert S.PRIMITIVA.fields["u"][1] == 56
    assert S.DATOS_MLP.itemsize == 112
    assert S.REGISTRO.itemsize == 232
    assert S.REGISTRO.fields["valido"][1] == 228
    assert S.CAMARA.itemsize == 112
    assert S.LUZ.itemsize == 40
    assert ctypes.sizeof(S.CTinyBVHD_GPU) == 24
    assert ctypes.sizeof(S.CImagenGPU) == 16


def test_reference_params():
    from tests.helpers import reference_params
    p = reference_params()
    assert (p.max_depth, p.rr_min_depth, p.shadow_mesh, p.tri_format, p.spp) == (20, 11, 0, 0, 1)


def test_entry_points_reject_bad_arguments(built):
    from tfg_b200 import _lib
    from tfg_b200.structs import CRenderParams
    with pytest.raises(_lib.TfgError) as e:
        _lib.call("tfgTraceRays", None, None, 0, None, 10, None, None)
    assert e.value.code == 10001 and "null" in _lib.last_error()
    with pytest.raises(_lib.TfgError):
        _lib.call("tfgRenderPass", None, None, None, 0, None, 0, 8, 8, 0, None, None, None, 0, None,
                  None, None, None, 0, None, None, 0, 0, None)
    p = CRenderParams()
    p.max_depth, p.spp = 0, 1
    with pytest.raises(_lib.TfgError):
        _lib.call("tfgRenderPass", ctypes.byref(p), 1, None, 0, None, 0, 8, 8, 0, None, None, None, 0, None,
                  None, None, None, 0, None, None, 0, 0, None)
    with pytest.raises(_lib.TfgError):
        _lib.call("tfgLaunchKernelComposite", None, None, None, 4, 4, None)
    # one-blob bins: a negative count is refused, an empty call does nothing
    with pytest.raises(_lib.TfgError) as e:
        _lib.call("tfgOneBlobBins", None, None, -1, None)
    assert e.value.code == 10001
    _lib.call("tfgOneBlobBins", None, None, 0, None)


def test_cwbvh_build_rejects_empty(built):
    from tfg_b200 import _lib
    from tfg_b200.structs import CCWBVHHost
    h = CCWBVHHost()
    with pytest.raises(_lib.TfgError):
        _lib.call("tfgCWBVHBuild", None, 0, ctypes.byref(h))


def test_tinybvh_construir_without_triangles_is_empty(built):
    from tfg_b200 import _lib, scenes
    from tfg_b200.structs import CTinyBVH
    prims = scenes.sphere_prim((0, 0, 0), 1.0)
    b = CTinyBVH()
    _lib.call("tfgTinyBVHConstruir", prims.ctypes.data, len(prims), ctypes.byref(b))
    assert b.num_primitivas == 0 and not b.ref.d_nodos
