"""Neural radiance cache model: the reference's ColorMLP (mlp.h:19-70) over
the native tensor-core kernels (tfgMlp* in include/tfg_pt.h)."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .structs import BOUNDS

N_PARAMS = 23552
# padded [out][in] shapes of the six weight matrices, in parameter order
LAYER_SHAPES = [(64, 96), (64, 64), (64, 64), (64, 64), (64, 64), (16, 64)]
WEIGHTS, EMA, ADAM_M, ADAM_V = 0, 1, 2, 3


def _stream(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def split_layers(flat: np.ndarray) -> list[np.ndarray]:
    out, o = [], 0
    for r, c in LAYER_SHAPES:
        out.append(flat[o:o + r * c].reshape(r, c))
        o += r * c
    return out


class ColorMLP:
    """ColorMLP(n_in=15, n_out=3, batch): train_step / inference / setBounds."""

    def __init__(self, n_in: int = 15, n_out: int = 3, batch: int = 16384, seed: int = 1337):
        self.batch = batch
        h = ctypes.c_void_p()
        _lib.call("tfgMlpCreate", n_in, n_out, batch, seed, ctypes.byref(h))
        self.h = h

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

    def inference_composite(self, datos: torch.Tensor, thr: torch.Tensor, img: torch.Tensor, n: int,
                            stream=None) -> None:
        _lib.call("tfgMlpInferenceComposite", self.h, datos.data_ptr(), thr.data_ptr(), img.data_ptr(), int(n),
                  _stream(stream))

    def get_params(self, which: int = WEIGHTS) -> np.ndarray:
        out = np.zeros(N_PARAMS, np.float32)
        _lib.call("tfgMlpGetParams", self.h, which, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), N_PARAMS)
        return out

    def set_params(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, np.float32)
        assert w.size == N_PARAMS
        _lib.call("tfgMlpSetParams", self.h, w.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), N_PARAMS)

    def compute_gradient(self, buffer: torch.Tensor, n_available: int, seed: int) -> tuple[np.ndarray, float]:
        g = np.zeros(N_PARAMS, np.float32)
        loss = ctypes.c_float(0.0)
        _lib.call("tfgMlpComputeGradient", self.h, buffer.data_ptr(), int(n_available), seed,
                  g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), N_PARAMS, ctypes.byref(loss))
        return g, float(loss.value)

    def save_model(self, path: str) -> None:
        """Weights, EMA and Adam moments as one float32 .npz archive."""
        np.savez(path, w=self.get_params(WEIGHTS), ema=self.get_params(EMA))

    def load_model(self, path: str) -> bool:
        try:
            d = np.load(path)
            self.set_params(d["ema"])
            return True
        except (OSError, KeyError, ValueError):
            return False


def status() -> None:
    _lib.call("tfgMlpStatus")
