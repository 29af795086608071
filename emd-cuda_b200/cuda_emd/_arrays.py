"""Array interop: accept torch (CUDA/CPU), CuPy (DLPack / CUDA array
interface) or NumPy arrays; hand device tensors to the C ABI; return results
in the caller's framework.  Never casts dtypes (the reference raises instead)."""
from __future__ import annotations

import numpy as np


def _torch():
    import torch
    return torch


def kind_of(x) -> str:
    torch = _torch()
    if isinstance(x, torch.Tensor):
        return "torch" if x.is_cuda else "torch_cpu"
    if isinstance(x, np.ndarray):
        return "numpy"
    if hasattr(x, "__cuda_array_interface__") or hasattr(x, "__dlpack__"):
        return "cupy"
    return "numpy"


def device_of(x, default: int) -> int:
    torch = _torch()
    if isinstance(x, torch.Tensor) and x.is_cuda:
        return x.device.index
    return default


def _to_torch(x, device: int):
    torch = _torch()
    k = kind_of(x)
    if k == "torch":
        t = x if x.device.index == device else x.to(f"cuda:{device}")
    elif k == "torch_cpu":
        t = x.to(f"cuda:{device}")
    elif k == "cupy":
        t = torch.from_dlpack(x)
        if t.device.index != device:
            t = t.to(f"cuda:{device}")
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(x))).to(f"cuda:{device}")
    return t.contiguous(), k


def as_device_f64(x, device: int):
    torch = _torch()
    t, k = _to_torch(x, device)
    if t.dtype != torch.float64:
        raise ValueError(f"expected float64, got {t.dtype}")
    return t, k


def as_device_real(x, device: int, f32: bool):
    """Device tensor of the launcher's value type (float64, or float32 for
    the FP32 kernels); any other dtype raises."""
    if not f32:
        return as_device_f64(x, device)
    torch = _torch()
    t, k = _to_torch(x, device)
    if t.dtype != torch.float32:
        raise ValueError(f"expected float32, got {t.dtype}")
    return t, k


def as_device_i64(x, device: int):
    torch = _torch()
    t, _ = _to_torch(x, device)
    if t.dtype != torch.int64:
        raise ValueError(f"offsets must be int64, got {t.dtype}")
    return t


def as_device_i32(x, device: int):
    torch = _torch()
    t, _ = _to_torch(x, device)
    if t.dtype != torch.int32:
        raise ValueError(f"order must be int32, got {t.dtype}")
    return t


def to_caller(t, kind: str):
    if kind == "torch":
        return t
    if kind == "torch_cpu":
        return t.cpu()
    if kind == "cupy":
        try:
            import cupy
            return cupy.from_dlpack(t)
        except ImportError:
            return t
    return t.cpu().numpy()


def stream_of(device) -> int:
    torch = _torch()
    return torch.cuda.current_stream(device).cuda_stream
