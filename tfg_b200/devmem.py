"""Zero-copy torch views of device memory owned by the native library."""
from __future__ import annotations

import numpy as np
import torch


class _CudaArray:
    def __init__(self, ptr: int, shape: tuple, typestr: str):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def view_device(ptr: int, count: int, dtype=np.float32, device="cuda") -> torch.Tensor:
    """A torch tensor aliasing `count` elements at device address `ptr`."""
    typestr = np.dtype(dtype).str
    return torch.as_tensor(_CudaArray(ptr, (int(count),), typestr), device=device)


def copy_from_device(dst: torch.Tensor, ptr: int) -> None:
    dst.copy_(view_device(ptr, dst.numel(), np.dtype(str(dst.dtype).replace("torch.", "")), dst.device))
