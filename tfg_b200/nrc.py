"""Neural radiance cache model: the reference's ColorMLP (mlp.h:19-70) over
the native tensor-core kernels (tfgMlp* in include/tfg_pt.h)."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .structs import (BOUNDS, DATOS_MLP, REGISTRO, CHashGridConfig, CMlpTuning, CNrcBuffers, CNrcFrameConfig,
                      CNrcSceneFrame)

def layer_shapes(hidden_layers: int = 5, width: int = 64) -> list[tuple[int, int]]:
    """Padded [out][in] shapes of the weight matrices, in parameter order."""
    return [(width, 96)] + [(width, width)] * (hidden_layers - 1) + [(16, width)]


def param_count(hidden_layers: int = 5, width: int = 64) -> int:
    return sum(r * c for r, c in layer_shapes(hidden_layers, width))


# the default network: 5 hidden layers of 64
LAYER_SHAPES = layer_shapes(5)
N_PARAMS = param_count(5)
WEIGHTS, EMA, ADAM_M, ADAM_V = 0, 1, 2, 3
FP16, BF16, FP8 = 0, 1, 2      # inference operand precisions (TFG_MLP_*)
FREQUENCY, HASHGRID = "frequency", "hashgrid"   # input encodings


def hashgrid_reference() -> dict:
    """The reference's hash-grid settings (mlp.cpp:33-39)."""
    c = CHashGridConfig()
    _lib.lib.tfgHashGridConfigReference(ctypes.byref(c))
    return {"n_levels": c.n_levels, "log2_hashmap_size": c.log2_hashmap_size,
            "base_resolution": c.base_resolution, "per_level_scale": c.per_level_scale}


def one_blob_bins(values: torch.Tensor, stream=None) -> torch.Tensor:
    """One-blob bins (4 per value) of a CUDA float32 tensor of values in
    [0, 1], as the composite encoding computes them (tfgOneBlobBins)."""
    if values.dtype != torch.float32 or not values.is_cuda or not values.is_contiguous():
        raise ValueError("one_blob_bins wants a contiguous float32 CUDA tensor")
    out = torch.empty(values.numel() * 4, dtype=torch.float32, device=values.device)
    _lib.call("tfgOneBlobBins", values.data_ptr(), out.data_ptr(), values.numel(), _stream(stream))
    return out.view(-1, 4)


def _stream(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def split_layers(flat: np.ndarray) -> list[np.ndarray]:
    """Weight matrices of a flat parameter array (its length gives the depth
    and the width)."""
    for width in (64, 128):
        hidden = (len(flat) - 112 * width) // (width * width) + 1
        if hidden >= 1 and param_count(hidden, width) == len(flat):
            break
    else:
        raise AssertionError("not a parameter array of this network")
    out, o = [], 0
    for r, c in layer_shapes(hidden, width):
        out.append(flat[o:o + r * c].reshape(r, c))
        o += r * c
    return out


class ColorMLP:
    """ColorMLP(n_in=15, n_out=3, batch): train_step / inference / setBounds.
    `hidden_layers` (3, 5 or 7; the reference's network has 5) sets the depth;
    `encoding` the input encoding: FREQUENCY, or HASHGRID, the reference's own
    composite (hash grid + one-blob + identity; `hashgrid` overrides fields of
    hashgrid_reference())."""

    def __init__(self, n_in: int = 15, n_out: int = 3, batch: int = 16384, seed: int = 1337, hidden_layers: int = 5,
                 encoding: str = FREQUENCY, hashgrid: dict | None = None, width: int = 64):
        self.batch = batch
        self.hidden_layers = hidden_layers
        self.encoding = encoding
        self.width = width
        h = ctypes.c_void_p()
        if encoding == HASHGRID:
            cfg = {**hashgrid_reference(), **(hashgrid or {})}
            c = CHashGridConfig()
            c.n_levels, c.log2_hashmap_size = cfg["n_levels"], cfg["log2_hashmap_size"]
            c.base_resolution, c.per_level_scale = cfg["base_resolution"], cfg["per_level_scale"]
            self.hashgrid = cfg
            _lib.call("tfgMlpCreateWide", n_in, n_out, batch, seed, hidden_layers, width, ctypes.byref(c),
                      ctypes.byref(h))
        elif encoding == FREQUENCY:
            self.hashgrid = None
            _lib.call("tfgMlpCreateWide", n_in, n_out, batch, seed, hidden_layers, width, None, ctypes.byref(h))
        else:
            raise ValueError(f"unknown encoding {encoding!r}")
        self.h = h
        self.n_params = int(_lib.lib.tfgMlpParamCount(self.h))
        self.n_table = int(_lib.lib.tfgMlpHashParamCount(self.h))

    def close(self) -> None:
        if self.h:
            _lib.lib.tfgMlpDestroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_bounds(self, lo, hi) -> None:
        b = np.zeros(1, BOUNDS)
        b["min"]["x"], b["min"]["y"], b["min"]["z"] = lo
        b["max"]["x"], b["max"]["y"], b["max"]["z"] = hi
        _lib.call("tfgMlpSetBounds", self.h, b.ctypes.data)

    def set_hyperparams(self, lr=1e-2, beta1=0.9, beta2=0.99, eps=1e-15, ema_decay=0.99) -> None:
        _lib.call("tfgMlpSetHyperparams", self.h, lr, beta1, beta2, eps, ema_decay)

    def train_step(self, buffer: torch.Tensor, n_available: int, read_loss: bool = True, stream=None) -> float:
        loss = ctypes.c_float(0.0)
        _lib.call("tfgMlpTrainStep", self.h, buffer.data_ptr(), int(n_available),
                  ctypes.byref(loss) if read_loss else None, _stream(stream))
        return float(loss.value)

    def inference(self, datos: torch.Tensor, out: torch.Tensor, n: int, stream=None) -> None:
        _lib.call("tfgMlpInference", self.h, datos.data_ptr(), out.data_ptr(), int(n), _stream(stream))

    def set_precision(self, precision: int) -> None:
        """Operand precision of later inference calls: FP16, BF16 or FP8."""
        _lib.call("tfgMlpSetPrecision", self.h, precision)

    def calibrate(self, datos: torch.Tensor, n: int, stream=None) -> None:
        """FP8 input scales from the per-layer amax of n samples."""
        _lib.call("tfgMlpCalibrate", self.h, datos.data_ptr(), n, _stream(stream))

    def set_tuning(self, wgrad_tiles_per_cta: int = 0, infer_ctas: int = 0) -> None:
        """Batch tiling of the model's kernels (0 = default)."""
        t = CMlpTuning()
        t.wgrad_tiles_per_cta, t.infer_ctas = wgrad_tiles_per_cta, infer_ctas
        _lib.call("tfgMlpTuningSet", self.h, ctypes.byref(t))

    def get_tuning(self) -> dict:
        t = CMlpTuning()
        _lib.call("tfgMlpTuningGet", self.h, ctypes.byref(t))
        return {"wgrad_tiles_per_cta": int(t.wgrad_tiles_per_cta), "infer_ctas": int(t.infer_ctas)}

    def autotune(self, datos: torch.Tensor | None = None, out: torch.Tensor | None = None, n: int = 0,
                 repeats: int = 5, stream=None) -> dict:
        """tfgMlpAutotune: weight-gradient tiles per CTA of one training batch
        and inference CTAs over `n` samples of `datos` (skipped when n = 0).
        The model state is left as it was; the winners are set and returned
        with their times."""
        t = CMlpTuning()
        ms = (ctypes.c_float * 2)()
        _lib.call("tfgMlpAutotune", self.h, datos.data_ptr() if datos is not None else None, int(n),
                  out.data_ptr() if out is not None else None, repeats, ctypes.byref(t), ms, _stream(stream))
        return {"wgrad_tiles_per_cta": int(t.wgrad_tiles_per_cta), "infer_ctas": int(t.infer_ctas),
                "wgrad_ms": float(ms[0]), "infer_ms": float(ms[1])}

    def encode_features(self, datos: torch.Tensor, n: int, training: bool = False, stream=None) -> torch.Tensor:
        """tfgMlpEncodeFeatures: the (n, 96) layer-0 operands the cache kernels
        compute for n queries -- the training forward pass's FP16 features, or
        inference's at the model's precision (FP16 / BF16)."""
        out = torch.empty(max(n, 1) * 96, dtype=torch.float32, device=datos.device)
        _lib.call("tfgMlpEncodeFeatures", self.h, datos.data_ptr(), int(n), 0 if training else 1, out.data_ptr(),
                  _stream(stream))
        return out[:n * 96].view(n, 96)

    def inference_composite(self, datos: torch.Tensor, thr: torch.Tensor, img: torch.Tensor, n: int,
                            stream=None) -> None:
        _lib.call("tfgMlpInferenceComposite", self.h, datos.data_ptr(), thr.data_ptr(), img.data_ptr(), int(n),
                  _stream(stream))

    def get_params(self, which: int = WEIGHTS) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        _lib.call("tfgMlpGetParams", self.h, which, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), self.n_params)
        return out

    def set_params(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, np.float32)
        assert w.size == self.n_params
        _lib.call("tfgMlpSetParams", self.h, w.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), self.n_params)

    def get_table(self, which: int = WEIGHTS) -> np.ndarray:
        """Hash-grid table array [level][entry][feature] (flat)."""
        out = np.zeros(self.n_table, np.float32)
        _lib.call("tfgMlpGetHashParams", self.h, which, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                  self.n_table)
        return out

    def set_table(self, t: np.ndarray) -> None:
        t = np.ascontiguousarray(t, np.float32)
        assert t.size == self.n_table
        _lib.call("tfgMlpSetHashParams", self.h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), self.n_table)

    def compute_gradient_ex(self, buffer: torch.Tensor, n_available: int,
                            seed: int) -> tuple[np.ndarray, np.ndarray, float]:
        """Gradients of the layer weights and of the hash-grid tables, and the loss."""
        g = np.zeros(self.n_params, np.float32)
        gt = np.zeros(self.n_table, np.float32)
        loss = ctypes.c_float(0.0)
        _lib.call("tfgMlpComputeGradientEx", self.h, buffer.data_ptr(), int(n_available), seed,
                  g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), self.n_params,
                  gt.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) if self.n_table else None, self.n_table,
                  ctypes.byref(loss))
        return g, gt, float(loss.value)

    def compute_gradient(self, buffer: torch.Tensor, n_available: int, seed: int) -> tuple[np.ndarray, float]:
        g = np.zeros(self.n_params, np.float32)
        loss = ctypes.c_float(0.0)
        _lib.call("tfgMlpComputeGradient", self.h, buffer.data_ptr(), int(n_available), seed,
                  g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), self.n_params, ctypes.byref(loss))
        return g, float(loss.value)

    def save_model(self, path: str) -> None:
        """Binary checkpoint (tfgMlpSave): weights, weight average, Adam state,
        counters, bounds and hyper-parameters."""
        _lib.call("tfgMlpSave", self.h, str(path).encode())

    def state(self) -> dict:
        st = (ctypes.c_uint32 * 8)()
        _lib.call("tfgMlpGetState", self.h, st)
        return {"step": st[0], "adam_t": st[1], "records": st[2], "gate": st[3],
                "loss_ema": float(np.array([st[4]], np.uint32).view(np.float32)[0])}

    def load_model(self, path: str) -> bool:
        """Restore a checkpoint written by save_model (same depth); False when
        the file is missing or not a checkpoint of this network, as the
        reference's load_model (mlp.cpp:196-276)."""
        try:
            _lib.call("tfgMlpLoad", self.h, str(path).encode())
            return True
        except _lib.TfgError:
            return False


def status() -> None:
    _lib.call("tfgMlpStatus")




class NrcRenderer:
    """The reference's normal-mode frame loop (main.cpp:895-1089) as GPU-only
    frames: tfgNrcFrame renders with cache queries and training records,
    answers and composites the queries, bootstraps targets and trains."""

    def __init__(self, ds, mlp: ColorMLP, params, train_steps: int = 4, max_records: int = 65536,
                 min_records: int = 1024, gate_threshold: float = 0.0, use_graph: bool = True, stream=None,
                 footprint: float | None = None, train_fraction: float | None = None):
        """`footprint` / `train_fraction` override the reference's cache
        policy (0.01 and 0.05, render.h:102 and :443); `gate_threshold` > 0
        turns on the per-cell gate judged by the path tracer."""
        self.ds, self.mlp, self.params = ds, mlp, params
        W, H = ds.scene.width, ds.scene.height
        dev = ds.device
        n = W * H
        self.W, self.H = W, H
        self.stream = stream or torch.cuda.Stream(device=dev)
        self.img = torch.zeros(n * 3, dtype=torch.float32, device=dev)
        self.accum = torch.zeros(n * 3, dtype=torch.float32, device=dev)
        self.infer = torch.zeros(n * DATOS_MLP.itemsize, dtype=torch.uint8, device=dev)
        self.thr = torch.zeros(n * 3, dtype=torch.float32, device=dev)
        self.ring_cap = max(n, max_records)
        self.regs = torch.zeros(self.ring_cap * REGISTRO.itemsize, dtype=torch.uint8, device=dev)
        self.counter = torch.zeros(1, dtype=torch.int32, device=dev)
        self.tail_in = torch.zeros(max_records * DATOS_MLP.itemsize, dtype=torch.uint8, device=dev)
        self.tail_pred = torch.zeros(max_records * 3, dtype=torch.float32, device=dev)
        self.train_buf = torch.zeros(max_records * DATOS_MLP.itemsize, dtype=torch.uint8, device=dev)
        self.cfg = CNrcFrameConfig()
        _lib.lib.tfgNrcFrameConfigReference(ctypes.byref(self.cfg))
        self.cfg.train_steps, self.cfg.max_records, self.cfg.min_records = train_steps, max_records, min_records
        self.cfg.gate_threshold, self.cfg.use_graph = gate_threshold, int(use_graph)
        if footprint is not None:
            self.cfg.footprint = footprint
        if train_fraction is not None:
            self.cfg.train_fraction = train_fraction
        self.bufs = CNrcBuffers(self.img.data_ptr(), self.accum.data_ptr(), self.infer.data_ptr(),
                                self.thr.data_ptr(), self.regs.data_ptr(), self.counter.data_ptr(), self.ring_cap, 0,
                                self.tail_in.data_ptr(), self.tail_pred.data_ptr(), self.train_buf.data_ptr())
        self.frames_accumulated = 0

    def frame(self, frame: int, warmup: bool = False, accumulate: bool = True) -> None:
        ds = self.ds
        self.cfg.warmup = int(warmup)
        self.bufs.accum = self.accum.data_ptr() if accumulate else None
        _lib.call("tfgNrcFrame", self.mlp.h, ctypes.byref(self.cfg), ctypes.byref(self.params.c()),
                  ds.camera.data_ptr(), ds.prims.data_ptr() if ds.prims is not None else None, ds.n_prims,
                  ds.lights.data_ptr(), ds.n_lights, self.W, self.H, ctypes.byref(ds.bvh.ref), ds.bvh.d_tris_wt,
                  ds.bvh.d_primitivas, ds.n_mesh, ctypes.byref(self.bufs), frame, self.stream.cuda_stream)
        if accumulate:
            self.frames_accumulated += 1

    def image(self) -> torch.Tensor:
        return self.img.view(self.H, self.W, 3)

    def mean_image(self) -> torch.Tensor:
        return (self.accum / max(1, self.frames_accumulated)).view(self.H, self.W, 3)

    def reset_accumulation(self) -> None:
        with torch.cuda.stream(self.stream):
            self.accum.zero_()
        self.frames_accumulated = 0


class NrcBatch:
    """Several independent scenes, each with its own cache model and
    NrcRenderer buffers, advanced one frame at a time by tfgNrcFrameBatch:
    up to four concurrent branches, optionally captured as one CUDA graph.
    No reference counterpart (the reference renders one scene per process)."""

    def __init__(self, renderers: list[NrcRenderer], use_graph: bool = True, stream=None):
        if not renderers:
            raise ValueError("NrcBatch needs at least one renderer")
        self.renderers = renderers
        self.use_graph = use_graph
        dev = renderers[0].ds.device
        self.stream = stream or torch.cuda.Stream(device=dev)
        n = len(renderers)
        self._arr = (CNrcSceneFrame * n)()
        self._params = [r.params.c() for r in renderers]

    def frame(self, frame: int, warmup: bool = False, accumulate: bool = False) -> None:
        for k, r in enumerate(self.renderers):
            r.cfg.warmup = int(warmup)
            r.bufs.accum = r.accum.data_ptr() if accumulate else None
            ds = r.ds
            f = self._arr[k]
            f.mlp = r.mlp.h
            f.cfg = ctypes.addressof(r.cfg)
            f.params = ctypes.addressof(self._params[k])
            f.camara = ds.camera.data_ptr()
            f.primitivas = ds.prims.data_ptr() if ds.prims is not None else None
            f.luces = ds.lights.data_ptr()
            f.bvh = ctypes.addressof(ds.bvh.ref)
            f.tris_wt = ds.bvh.d_tris_wt
            f.primitivas_bvh = ds.bvh.d_primitivas
            f.buffers = ctypes.addressof(r.bufs)
            f.num_primitivas, f.num_luces, f.num_prims_bvh = ds.n_prims, ds.n_lights, ds.n_mesh
            f.ancho_img, f.alto_img = r.W, r.H
            if accumulate:
                r.frames_accumulated += 1
        _lib.call("tfgNrcFrameBatch", len(self.renderers), self._arr, frame, int(self.use_graph),
                  self.stream.cuda_stream)


def reconstruct(ds, mlp: ColorMLP, params, spp: int, first_frame: int = 0, stream=None) -> torch.Tensor:
    """The reference's reconstruction mode (tfgNrcReconstruct): `spp` samples
    answered by a trained cache without training; returns the (H*W*3) sum."""
    W, H = ds.scene.width, ds.scene.height
    n = W * H
    dev = ds.device
    img = torch.zeros(n * 3, dtype=torch.float32, device=dev)
    infer = torch.zeros(n * DATOS_MLP.itemsize, dtype=torch.uint8, device=dev)
    thr = torch.zeros(n * 3, dtype=torch.float32, device=dev)
    accum = torch.empty(n * 3, dtype=torch.float32, device=dev)
    _lib.call("tfgNrcReconstruct", mlp.h, ctypes.byref(params.c()), ds.camera.data_ptr(),
              ds.prims.data_ptr() if ds.prims is not None else None, ds.n_prims, ds.lights.data_ptr(), ds.n_lights,
              W, H, ctypes.byref(ds.bvh.ref), ds.bvh.d_tris_wt, ds.bvh.d_primitivas, ds.n_mesh, spp, first_frame,
              img.data_ptr(), infer.data_ptr(), thr.data_ptr(), accum.data_ptr(), _stream(stream))
    return accum
