"""Host-side API over the C ABI: the reference's render call sequence
(main.cpp:822-1016) as Python objects.

``DeviceScene`` uploads a :class:`~tfg_b200.scenes.Scene` and builds its CWBVH
(``tfgTinyBVHConstruir``, the drop-in for TinyBVH::construirBVH).  The render
functions call ``tfgLaunchKernelRenderTiny`` / ``tfgRenderPass``.  torch is
used only to own device memory and to name the stream.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .scenes import Scene
from .structs import (CImagenGPU, CRenderParams, CRenderProfile, CRenderScene, CRenderTuning, CTinyBVH,
                      CTinyBVHD_GPU, CTuneRecord, DATOS_MLP, REGISTRO)

TRIS_REF, TRIS_WATERTIGHT = 0, 1
PROFILE_TIMES, PROFILE_COUNTS = 1, 2
STAGES = ("generate", "trace", "shade", "shadow", "resolve")


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _stream(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def _dev_bytes(arr: np.ndarray, device) -> torch.Tensor | None:
    if arr is None or len(arr) == 0:
        return None
    return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).copy()).to(device)


@dataclass
class RenderParams:
    max_depth: int = 20          # render.h:63
    rr_min_depth: int = 11       # render.h:209 (depth > 10)
    shadow_mesh: int = 0         # escenario.h:65,168 (mesh never occludes in the reference kernel)
    tri_format: int = TRIS_REF
    spp: int = 1
    accumulate: int = 0
    profile: int = 0             # PROFILE_TIMES | PROFILE_COUNTS

    @staticmethod
    def reference() -> "RenderParams":
        return RenderParams()

    def c(self) -> CRenderParams:
        p = CRenderParams()
        p.max_depth, p.rr_min_depth, p.shadow_mesh = self.max_depth, self.rr_min_depth, self.shadow_mesh
        p.tri_format, p.spp, p.accumulate = self.tri_format, self.spp, self.accumulate
        p.profile = self.profile
        return p


class DeviceScene:
    """Scene resident on a GPU: analytic primitives, lights, camera, CWBVH."""

    def __init__(self, scene: Scene, device="cuda", gpu_build: bool = False):
        """`gpu_build`: build the CWBVH on the device (tfgTinyBVHConstruirGPU,
        Morton-order tree) instead of the host binned-SAH builder."""
        self.scene = scene
        self.device = torch.device(device)
        self.prims = _dev_bytes(scene.prims, self.device)
        self.lights = _dev_bytes(scene.lights, self.device)
        self.camera = _dev_bytes(scene.camera, self.device)
        self.bvh = CTinyBVH()
        mesh = np.ascontiguousarray(scene.mesh)
        with torch.cuda.device(self.device):
            if gpu_build:
                dmesh = _dev_bytes(mesh, self.device)
                _lib.call("tfgTinyBVHConstruirGPU", _ptr(dmesh), len(mesh), ctypes.byref(self.bvh),
                          _stream(None))
                del dmesh
            else:
                _lib.call("tfgTinyBVHConstruir", mesh.ctypes.data if len(mesh) else None, len(mesh),
                          ctypes.byref(self.bvh))
        self.n_prims = len(scene.prims)
        self.n_lights = len(scene.lights)
        self.n_mesh = int(self.bvh.num_primitivas)

    def set_camera(self, cam: np.ndarray) -> None:
        self.camera.copy_(torch.from_numpy(np.ascontiguousarray(cam).view(np.uint8).copy()))

    @property
    def ref_bvh(self) -> CTinyBVHD_GPU:
        return self.bvh.ref

    def close(self) -> None:
        if self.bvh.ref.d_nodos:
            _lib.lib.tfgTinyBVHLiberar(ctypes.byref(self.bvh))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NrcBuffers:
    """Per-pixel cache-query / throughput buffers and the training-record ring
    (main.cpp:908-930)."""

    def __init__(self, n_pixels: int, device, ring_cap: int | None = None):
        self.n = n_pixels
        self.cap = ring_cap or n_pixels
        self.infer = torch.zeros(n_pixels * DATOS_MLP.itemsize, dtype=torch.uint8, device=device)
        self.thr = torch.zeros(n_pixels * 3, dtype=torch.float32, device=device)
        self.regs = torch.zeros(self.cap * REGISTRO.itemsize, dtype=torch.uint8, device=device)
        self.counter = torch.zeros(1, dtype=torch.int32, device=device)


def render_reference_call(ds: DeviceScene, frame: int, img: torch.Tensor, nrc: NrcBuffers | None = None,
                          use_inf: bool = False, train: bool = False, stream=None) -> None:
    """tfgLaunchKernelRenderTiny with the reference's arguments: one sample per
    pixel into `img` (H*W*3 floats)."""
    W, H = ds.scene.width, ds.scene.height
    im = CImagenGPU(W, H, img.data_ptr())
    thr = nrc.thr if nrc is not None else torch.zeros(W * H * 3, dtype=torch.float32, device=img.device)
    _lib.call("tfgLaunchKernelRenderTiny",
              _ptr(ds.camera), _ptr(ds.prims), ds.n_prims, _ptr(ds.lights), ds.n_lights, None, 0, W, H, 1, frame,
              ctypes.byref(ds.bvh.ref), ds.bvh.d_primitivas, ds.n_mesh, ctypes.byref(im), None,
              _ptr(nrc.regs) if nrc else None, _ptr(nrc.counter) if nrc else None, nrc.cap if nrc else 0,
              _ptr(nrc.infer) if nrc else None, _ptr(thr), int(use_inf), int(train), _stream(stream))


def render_pass(ds: DeviceScene, params: RenderParams, frame: int, img: torch.Tensor | None = None,
                accum: torch.Tensor | None = None, nrc: NrcBuffers | None = None, use_inf: bool = False,
                train: bool = False, stream=None) -> None:
    """tfgRenderPass: params.spp samples (frames frame..frame+spp-1); `accum`
    (H*W*3 floats) receives the sum when params.accumulate is set."""
    W, H = ds.scene.width, ds.scene.height
    im = CImagenGPU(W, H, img.data_ptr() if img is not None else None)
    _lib.call("tfgRenderPass", ctypes.byref(params.c()),
              _ptr(ds.camera), _ptr(ds.prims), ds.n_prims, _ptr(ds.lights), ds.n_lights, W, H, frame,
              ctypes.byref(ds.bvh.ref), ds.bvh.d_tris_wt, ds.bvh.d_primitivas, ds.n_mesh, ctypes.byref(im),
              _ptr(accum), _ptr(nrc.regs) if nrc else None, _ptr(nrc.counter) if nrc else None,
              nrc.cap if nrc else 0, _ptr(nrc.infer) if nrc else None, _ptr(nrc.thr) if nrc else None,
              int(use_inf), int(train), _stream(stream))


def render_pass_batch(dss: list, params: RenderParams, frame: int, imgs: list | None = None,
                      accums: list | None = None, stream=None) -> None:
    """tfgRenderPassBatch: plain path tracing of several scenes, each stage
    launched once for all of them; imgs / accums: per scene (or None)."""
    n = len(dss)
    arr = (CRenderScene * n)()
    for k, ds in enumerate(dss):
        f = arr[k]
        f.camara, f.primitivas, f.num_primitivas = _ptr(ds.camera), _ptr(ds.prims), ds.n_prims
        f.luces, f.num_luces = _ptr(ds.lights), ds.n_lights
        f.ancho_img, f.alto_img = ds.scene.width, ds.scene.height
        f.nodos_bvh = ctypes.addressof(ds.bvh.ref)
        f.tris_wt, f.primitivas_bvh, f.num_prims_bvh = ds.bvh.d_tris_wt, ds.bvh.d_primitivas, ds.n_mesh
        f.imagen = _ptr(imgs[k]) if imgs is not None else None
        f.accum = _ptr(accums[k]) if accums is not None else None
    _lib.call("tfgRenderPassBatch", n, arr, ctypes.byref(params.c()), frame, _stream(stream))


def render_pass_static(ds: DeviceScene, params: RenderParams, frame: int, img: torch.Tensor | None = None,
                       accum: torch.Tensor | None = None, stream=None) -> None:
    """tfgRenderPassStatic: the same pass with no device allocation (plain path
    tracing, at most 16384 pixels; calls must not overlap on the GPU)."""
    W, H = ds.scene.width, ds.scene.height
    im = CImagenGPU(W, H, img.data_ptr() if img is not None else None)
    _lib.call("tfgRenderPassStatic", ctypes.byref(params.c()),
              _ptr(ds.camera), _ptr(ds.prims), ds.n_prims, _ptr(ds.lights), ds.n_lights, W, H, frame,
              ctypes.byref(ds.bvh.ref), ds.bvh.d_tris_wt, ds.bvh.d_primitivas, ds.n_mesh, ctypes.byref(im),
              _ptr(accum), _stream(stream))


def camera_rays(ds: DeviceScene, frame: int, rays: torch.Tensor, stream=None) -> None:
    W, H = ds.scene.width, ds.scene.height
    _lib.call("tfgGenerateCameraRays", _ptr(ds.camera), W, H, frame, _ptr(rays), _stream(stream))


RAYS_SCANLINE, RAYS_TILES = 0, 1


def camera_rays_ex(ds: DeviceScene, frame: int, samples: int, order: int, rays: torch.Tensor, stream=None) -> None:
    """tfgGenerateCameraRaysEx: `samples` samples of camera rays, sample-major,
    scanline or 8 x 4 tile order (rays: samples*W*H*8 floats)."""
    W, H = ds.scene.width, ds.scene.height
    _lib.call("tfgGenerateCameraRaysEx", _ptr(ds.camera), W, H, frame, samples, order, _ptr(rays), _stream(stream))


def tiled_pixels(W: int, H: int) -> np.ndarray:
    """Pixel index of every position of a sample in tile order (tfgTiledPixel)."""
    return np.array([_lib.lib.tfgTiledPixel(i, W, H) for i in range(W * H)], dtype=np.int64)


def trace_rays(ds: DeviceScene, rays: torch.Tensor, hits: torch.Tensor, tri_format: int = TRIS_WATERTIGHT,
               stream=None) -> None:
    n = rays.numel() // 8
    _lib.call("tfgTraceRays", ctypes.byref(ds.bvh.ref), ds.bvh.d_tris_wt, tri_format, _ptr(rays), n, _ptr(hits),
              _stream(stream))


def accumulate_spp(ds: DeviceScene, params: RenderParams, spp: int, first_frame: int = 0, stream=None) -> torch.Tensor:
    """Mean of `spp` samples per pixel as an (H, W, 3) float tensor."""
    W, H = ds.scene.width, ds.scene.height
    acc = torch.zeros(H * W * 3, dtype=torch.float32, device=ds.device)
    p = RenderParams(**{**params.__dict__, "spp": spp, "accumulate": 1})
    render_pass(ds, p, first_frame, None, acc, stream=stream)
    return (acc / spp).view(H, W, 3)


def tonemap_filmic(accum: torch.Tensor, frames: int, W: int, H: int, stream=None) -> tuple[torch.Tensor, torch.Tensor]:
    """tfgToneMapFilmic: the averaged HDR image (H, W, 3 float32) and the
    reference's filmic 8-bit image (H, W, 3 uint8), both on the device."""
    hdr = torch.empty(H * W * 3, dtype=torch.float32, device=accum.device)
    rgb8 = torch.empty(H * W * 3, dtype=torch.uint8, device=accum.device)
    _lib.call("tfgToneMapFilmic", _ptr(accum), frames, W, H, _ptr(hdr), _ptr(rgb8), _stream(stream))
    return hdr.view(H, W, 3), rgb8.view(H, W, 3)


def write_ppm(path: str, rgb8) -> None:
    """Binary PPM from an (H, W, 3) uint8 array or tensor (host copy made here)."""
    a = np.ascontiguousarray(rgb8.cpu().numpy() if isinstance(rgb8, torch.Tensor) else rgb8, dtype=np.uint8)
    _lib.call("tfgWritePPM", str(path).encode(), a.ctypes.data, a.shape[1], a.shape[0])


def write_pfm(path: str, rgb) -> None:
    """PFM (little-endian float RGB) from an (H, W, 3) float array or tensor."""
    a = np.ascontiguousarray(rgb.cpu().numpy() if isinstance(rgb, torch.Tensor) else rgb, dtype=np.float32)
    _lib.call("tfgWritePFM", str(path).encode(), a.ctypes.data, a.shape[1], a.shape[0])


def profile_reset() -> None:
    _lib.call("tfgRenderProfileReset")


def profile_get() -> dict:
    """Stage times (ms, launches) and traversal work since profile_reset()."""
    p = CRenderProfile()
    _lib.call("tfgRenderProfileGet", ctypes.byref(p))
    return {
        "ms": {k: p.ms[i] for i, k in enumerate(STAGES)},
        "launches": {k: int(p.launches[i]) for i, k in enumerate(STAGES)},
        "rays": int(p.rays), "nodes": int(p.nodes), "tri_tests": int(p.tri_tests),
        "shadow_rays": int(p.shadow_rays), "shadow_nodes": int(p.shadow_nodes),
        "shadow_tri_tests": int(p.shadow_tri_tests),
    }


@dataclass
class RenderTuning:
    """TfgRenderTuning: how the wavefront stages are sized and launched on the
    current device.  Every setting renders the same image."""
    wavefront_paths: int = 0      # queue capacity in paths; 0 = one sample of the image (W*H)
    trace_threads: int = 128      # threads per traversal / shadow CTA: 64, 128, 256
    trace_warps_per_sm: int = 0   # resident traversal warps per SM; 0 = as many as fit
    refill_min: int = 8           # idle lanes that make a traversal warp fetch new rays
    shadow_one_lane: int = 0      # 1: one lane traces all lights of a shading point
    refill_min_primary: int = 0   # first-bounce refill threshold; 0 = refill_min
    overlap_shadow: int = 1       # 1: shadow stage on a second stream beside the next trace

    def c(self) -> CRenderTuning:
        t = CRenderTuning()
        t.wavefront_paths, t.trace_threads, t.trace_warps_per_sm = (self.wavefront_paths, self.trace_threads,
                                                                    self.trace_warps_per_sm)
        t.refill_min, t.shadow_one_lane = self.refill_min, self.shadow_one_lane
        t.refill_min_primary, t.overlap_shadow = self.refill_min_primary, self.overlap_shadow
        return t

    @staticmethod
    def of(t: CRenderTuning) -> "RenderTuning":
        return RenderTuning(int(t.wavefront_paths), int(t.trace_threads), int(t.trace_warps_per_sm),
                            int(t.refill_min), int(t.shadow_one_lane), int(t.refill_min_primary),
                            int(t.overlap_shadow))

    @staticmethod
    def default() -> "RenderTuning":
        t = CRenderTuning()
        _lib.lib.tfgRenderTuningDefault(ctypes.byref(t))
        return RenderTuning.of(t)


def set_tuning(t: RenderTuning) -> None:
    _lib.call("tfgRenderTuningSet", ctypes.byref(t.c()))


def get_tuning() -> RenderTuning:
    t = CRenderTuning()
    _lib.call("tfgRenderTuningGet", ctypes.byref(t))
    return RenderTuning.of(t)


def autotune(ds: DeviceScene, params: RenderParams, repeats: int = 3, max_records: int = 64,
             stream=None) -> tuple[RenderTuning, list[tuple[RenderTuning, float]]]:
    """tfgRenderAutotune on this scene: sets and returns the fastest tuning and
    every candidate timed, as (tuning, ms per pass) in the order timed."""
    W, H = ds.scene.width, ds.scene.height
    out = CRenderTuning()
    recs = (CTuneRecord * max_records)()
    n = ctypes.c_int32(0)
    _lib.call("tfgRenderAutotune", ctypes.byref(params.c()), _ptr(ds.camera), _ptr(ds.prims), ds.n_prims,
              _ptr(ds.lights), ds.n_lights, W, H, ctypes.byref(ds.bvh.ref), ds.bvh.d_tris_wt, ds.bvh.d_primitivas,
              ds.n_mesh, repeats, ctypes.byref(out), recs, max_records, ctypes.byref(n), _stream(stream))
    table = [(RenderTuning.of(recs[i].tuning), float(recs[i].ms)) for i in range(min(n.value, max_records))]
    return RenderTuning.of(out), table
