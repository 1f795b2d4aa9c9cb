"""ctypes binding of the native library (tfg_b200/libtfgpt.so).

The library is the product: there is no Python or CPU fallback.  Importing
this module raises if the library has not been built.  Every wrapper below
raises ``TfgError`` on a non-zero return, carrying tfgGetLastErrorString().
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_float, c_int32, c_uint32, c_uint64, c_void_p
from pathlib import Path

from .structs import (CCWBVHHost, CHashGridConfig, CImagenGPU, CMlpTuning, CNrcBuffers, CNrcFrameConfig, CNrcSceneFrame,
                      CRenderParams, CRenderProfile, CRenderScene, CRenderTuning, CTinyBVH, CTinyBVHD_GPU,
                      CTuneRecord)

LIB_PATH = Path(__file__).resolve().parent / "libtfgpt.so"


class TfgError(RuntimeError):
    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed ({code}): {msg}")
        self.code = code


def _load() -> ctypes.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"native library missing: {LIB_PATH} (run tfg_b200/_build.py)")
    return ctypes.CDLL(str(LIB_PATH))


lib = _load()

# name -> (restype, argtypes)
_PROTOS = {
    "tfgGetLastErrorString": (c_char_p, []),
    "tfgCWBVHBuild": (c_int32, [POINTER(c_float), c_uint32, POINTER(CCWBVHHost)]),
    "tfgCWBVHFree": (None, [POINTER(CCWBVHHost)]),
    "tfgTinyBVHConstruir": (c_int32, [c_void_p, c_int32, POINTER(CTinyBVH)]),
    "tfgTinyBVHConstruirGPU": (c_int32, [c_void_p, c_int32, POINTER(CTinyBVH), c_void_p]),
    "tfgTinyBVHLiberar": (None, [POINTER(CTinyBVH)]),
    "tfgRenderParamsReference": (None, [POINTER(CRenderParams)]),
    "tfgRenderProfileReset": (c_int32, []),
    "tfgRenderProfileGet": (c_int32, [POINTER(CRenderProfile)]),
    "tfgRenderPassBatch": (c_int32, [c_int32, POINTER(CRenderScene), POINTER(CRenderParams), c_int32, c_void_p]),
    "tfgRenderTuningDefault": (None, [POINTER(CRenderTuning)]),
    "tfgRenderTuningSet": (c_int32, [POINTER(CRenderTuning)]),
    "tfgRenderTuningGet": (c_int32, [POINTER(CRenderTuning)]),
    "tfgRenderAutotune": (c_int32, [
        POINTER(CRenderParams), c_void_p, c_void_p, c_int32, c_void_p, c_int32, c_int32, c_int32,
        POINTER(CTinyBVHD_GPU), c_void_p, c_void_p, c_int32, c_int32, POINTER(CRenderTuning), POINTER(CTuneRecord),
        c_int32, POINTER(c_int32), c_void_p]),
    "tfgHashGridConfigReference": (None, [POINTER(CHashGridConfig)]),
    "tfgMlpCreateHashGrid": (c_int32, [c_uint32, c_uint32, c_uint32, c_uint64, c_int32, POINTER(CHashGridConfig),
                                       c_void_p]),
    "tfgMlpHashParamCount": (ctypes.c_int64, [c_void_p]),
    "tfgOneBlobBins": (c_int32, [c_void_p, c_void_p, c_int32, c_void_p]),
    "tfgMlpEncodeFeatures": (c_int32, [c_void_p, c_void_p, c_uint32, c_int32, c_void_p, c_void_p]),
    "tfgMlpCreateWide": (c_int32, [c_uint32, c_uint32, c_uint32, c_uint64, c_int32, c_int32, POINTER(CHashGridConfig),
                                   c_void_p]),
    "tfgMlpGetHashParams": (c_int32, [c_void_p, c_int32, POINTER(c_float), ctypes.c_int64]),
    "tfgMlpSetHashParams": (c_int32, [c_void_p, POINTER(c_float), ctypes.c_int64]),
    "tfgMlpComputeGradientEx": (c_int32, [c_void_p, c_void_p, c_uint32, c_uint32, POINTER(c_float), c_uint32,
                                          POINTER(c_float), ctypes.c_int64, POINTER(c_float)]),
    "tfgMlpTuningSet": (c_int32, [c_void_p, POINTER(CMlpTuning)]),
    "tfgMlpTuningGet": (c_int32, [c_void_p, POINTER(CMlpTuning)]),
    "tfgMlpAutotune": (c_int32, [c_void_p, c_void_p, c_uint32, c_void_p, c_int32, POINTER(CMlpTuning),
                                 POINTER(c_float), c_void_p]),
    "tfgLaunchKernelRenderTiny": (c_int32, [
        c_void_p, c_void_p, c_int32, c_void_p, c_int32, c_void_p, c_int32, c_int32, c_int32, c_int32, c_int32,
        POINTER(CTinyBVHD_GPU), c_void_p, c_int32, POINTER(CImagenGPU), c_void_p, c_void_p, c_void_p, c_int32,
        c_void_p, c_void_p, c_int32, c_int32, c_void_p]),
    "tfgRenderPass": (c_int32, [
        POINTER(CRenderParams), c_void_p, c_void_p, c_int32, c_void_p, c_int32, c_int32, c_int32, c_int32,
        POINTER(CTinyBVHD_GPU), c_void_p, c_void_p, c_int32, POINTER(CImagenGPU), c_void_p, c_void_p, c_void_p,
        c_int32, c_void_p, c_void_p, c_int32, c_int32, c_void_p]),
    "tfgRenderPassStatic": (c_int32, [
        POINTER(CRenderParams), c_void_p, c_void_p, c_int32, c_void_p, c_int32, c_int32, c_int32, c_int32,
        POINTER(CTinyBVHD_GPU), c_void_p, c_void_p, c_int32, POINTER(CImagenGPU), c_void_p, c_void_p]),
    "tfgTraceRays": (c_int32, [POINTER(CTinyBVHD_GPU), c_void_p, c_int32, c_void_p, c_int32, c_void_p, c_void_p]),
    "tfgGenerateCameraRays": (c_int32, [c_void_p, c_int32, c_int32, c_int32, c_void_p, c_void_p]),
    "tfgGenerateCameraRaysEx": (c_int32, [c_void_p, c_int32, c_int32, c_int32, c_int32, c_int32, c_void_p, c_void_p]),
    "tfgTiledPixel": (c_uint32, [c_uint32, c_uint32, c_uint32]),
    "tfgLaunchInicializarCamara": (c_int32, [c_void_p, c_int32, c_int32, c_void_p]),
    "tfgLaunchKernelComposite": (c_int32, [c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p]),
    "tfgLaunchKernelCalcularTargets": (c_int32, [c_void_p, c_void_p, c_void_p, c_int32, c_void_p]),
    "tfgLaunchKernelPrepararInferenciaTail": (c_int32, [c_void_p, c_void_p, c_int32, c_void_p]),
    "tfgLaunchGenerarIndicesAleatorios": (c_int32, [c_void_p, c_int32, c_int32, c_uint32, c_void_p]),
    "tfgLaunchPrepararDatosEntrenamiento": (c_int32, [c_void_p, c_void_p, c_int32, c_int32, c_int32, c_void_p,
                                                      c_void_p, c_void_p, c_void_p]),
    "tfgLaunchPrepararDatosInferencia": (c_int32, [c_void_p, c_uint32, c_uint32, c_void_p, c_void_p, c_void_p]),
    "tfgLaunchGuardarSalidaInferencia": (c_int32, [c_void_p, c_void_p, c_int32, c_void_p]),
    "tfgMlpCreate": (c_int32, [c_uint32, c_uint32, c_uint32, c_uint64, POINTER(c_void_p)]),
    "tfgMlpDestroy": (None, [c_void_p]),
    "tfgMlpSetBounds": (c_int32, [c_void_p, c_void_p]),
    "tfgMlpSetHyperparams": (c_int32, [c_void_p, c_float, c_float, c_float, c_float, c_float]),
    "tfgMlpTrainStep": (c_int32, [c_void_p, c_void_p, c_uint32, POINTER(c_float), c_void_p]),
    "tfgMlpInference": (c_int32, [c_void_p, c_void_p, c_void_p, c_uint32, c_void_p]),
    "tfgMlpCreateEx": (c_int32, [c_uint32, c_uint32, c_uint32, c_uint64, c_int32, c_void_p]),
    "tfgMlpParamCount": (c_int32, [c_void_p]),
    "tfgMlpSave": (c_int32, [c_void_p, c_char_p]),
    "tfgMlpLoad": (c_int32, [c_void_p, c_char_p]),
    "tfgNrcReconstruct": (c_int32, [c_void_p, POINTER(CRenderParams), c_void_p, c_void_p, c_int32, c_void_p, c_int32,
                                    c_int32, c_int32, POINTER(CTinyBVHD_GPU), c_void_p, c_void_p, c_int32, c_int32,
                                    c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "tfgToneMapFilmic": (c_int32, [c_void_p, c_int32, c_int32, c_int32, c_void_p, c_void_p, c_void_p]),
    "tfgWritePPM": (c_int32, [c_char_p, c_void_p, c_int32, c_int32]),
    "tfgWritePFM": (c_int32, [c_char_p, c_void_p, c_int32, c_int32]),
    "tfgMlpSelfTestWait": (c_int32, [c_uint32]),
    "tfgL2GatherPass": (c_int32, [c_void_p, c_uint32, c_uint32, c_uint32, c_void_p, c_int32, c_void_p]),
    "tfgMlpSetPrecision": (c_int32, [c_void_p, c_int32]),
    "tfgMlpCalibrate": (c_int32, [c_void_p, c_void_p, c_uint32, c_void_p]),
    "tfgMlpInferenceComposite": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_uint32, c_void_p]),
    "tfgMlpGetParams": (c_int32, [c_void_p, c_int32, POINTER(c_float), c_uint32]),
    "tfgMlpSetParams": (c_int32, [c_void_p, POINTER(c_float), c_uint32]),
    "tfgMlpComputeGradient": (c_int32, [c_void_p, c_void_p, c_uint32, c_uint32, POINTER(c_float), c_uint32,
                                        POINTER(c_float)]),
    "tfgMlpStatus": (c_int32, []),
    "tfgMlpGetState": (c_int32, [c_void_p, POINTER(c_uint32)]),
    "tfgNrcFrameConfigReference": (None, [POINTER(CNrcFrameConfig)]),
    "tfgNrcFrameBatch": (c_int32, [c_int32, POINTER(CNrcSceneFrame), c_int32, c_int32, c_void_p]),
    "tfgNrcFrame": (c_int32, [c_void_p, POINTER(CNrcFrameConfig), POINTER(CRenderParams), c_void_p, c_void_p, c_int32,
                              c_void_p, c_int32, c_int32, c_int32, POINTER(CTinyBVHD_GPU), c_void_p, c_void_p, c_int32,
                              POINTER(CNrcBuffers), c_int32, c_void_p]),
}

for _name, (_res, _args) in _PROTOS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def last_error() -> str:
    return lib.tfgGetLastErrorString().decode(errors="replace")


def check(fn: str, code: int) -> None:
    if code != 0:
        raise TfgError(fn, code, last_error())


def call(name: str, *args) -> None:
    check(name, getattr(lib, name)(*args))


def exported_symbols() -> list[str]:
    return list(_PROTOS)
