"""Device-buffer helpers: torch CUDA tensors are the only memory the Python
layer hands to libfastwigner (as raw pointers)."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import FastWignerError


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise FastWignerError("fastwigner_b200 needs a CUDA device (sm_100a); there is no CPU fallback")
    return torch.device("cuda", torch.cuda.current_device())


def ptr(t) -> ctypes.c_void_p:
    if t is None:
        return ctypes.c_void_p(0)
    return ctypes.c_void_p(t.data_ptr())


def stream_handle() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def to_device(a, dtype, device) -> torch.Tensor:
    """numpy/torch/scalar -> contiguous device tensor of `dtype`."""
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=dtype).contiguous()
    return torch.from_numpy(np.array(a, copy=True, order="C")).to(device=device, dtype=dtype).contiguous()


class DeviceArray:
    """Minimal gpuarray-like view of a device tensor, as returned by the
    CUDA-class drop-ins (the reference returned pycuda GPUArrays): ``.get()``
    copies to a numpy array, ``.tensor`` is the live device tensor."""

    def __init__(self, tensor: torch.Tensor):
        self.tensor = tensor

    def get(self) -> np.ndarray:
        return self.tensor.detach().cpu().numpy()

    @property
    def shape(self):
        return tuple(self.tensor.shape)

    @property
    def dtype(self):
        return np.dtype(str(self.tensor.dtype).replace("torch.", ""))

    @property
    def real(self):
        return DeviceArray(self.tensor.real if self.tensor.is_complex() else self.tensor)

    def copy(self):
        return DeviceArray(self.tensor.clone())

    def __array__(self, dtype=None, copy=None):
        a = self.get()
        return a if dtype is None else a.astype(dtype)

    def __repr__(self):
        return f"DeviceArray(shape={self.shape}, dtype={self.dtype})"
