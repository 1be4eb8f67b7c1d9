"""Device-array helpers: CUDA tensors that also answer CuPy's ``.get()``.

The reference returns CuPy arrays and calls ``.get()`` on them (``main/timestep.py:85``,
``main/timestep.py:102``, ``main/main.py:135``); the classes of this package return
``CudaArray`` tensors, a ``torch.Tensor`` subclass with the same ``.get()``.
"""
from __future__ import annotations

import numpy as np
import torch


class CudaArray(torch.Tensor):
    """torch.Tensor with CuPy's ``get()`` (device -> host NumPy copy)."""

    def get(self):
        return self.detach().to("cpu").numpy()


def device():
    if not torch.cuda.is_available():
        raise RuntimeError("vlasov1d2v_b200 needs a CUDA device (there is no CPU path)")
    return torch.device("cuda", torch.cuda.current_device())


def wrap(t):
    if isinstance(t, CudaArray):
        return t
    return t.as_subclass(CudaArray)


def plain(t):
    """The tensor without the subclass (cheaper for internal arithmetic)."""
    return t.as_subclass(torch.Tensor) if isinstance(t, CudaArray) else t


def as_tensor(x, dtype=None):
    """A contiguous CUDA tensor view/copy of ``x`` (NumPy array, tensor or scalar)."""
    if isinstance(x, torch.Tensor):
        t = plain(x)
        if t.device.type != "cuda":
            t = t.to(device())
        if dtype is not None and t.dtype != dtype:
            t = t.to(dtype)
        return t
    arr = np.asarray(x)
    if np.iscomplexobj(arr):
        t = torch.as_tensor(np.ascontiguousarray(arr), device=device())
    else:
        t = torch.as_tensor(np.ascontiguousarray(arr), dtype=dtype or torch.float64, device=device())
    return t


def const(owner, name, arr, complex_=False):
    """Cached device copy of a host table attached to ``owner``."""
    cache = owner.__dict__.setdefault("_dev_tables", {})
    key = (name, torch.cuda.current_device())
    if key not in cache:
        a = np.asarray(arr)
        dt = torch.complex128 if complex_ else (torch.float64 if a.dtype.kind == "f" else torch.int64)
        cache[key] = wrap(torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=device()))
    return cache[key]


def precision_of(t):
    if t.dtype == torch.float64:
        return "fp64"
    if t.dtype == torch.float32:
        return "fp32"
    raise TypeError(f"state dtype {t.dtype} is not supported (float64 or float32)")


def stream_handle():
    return torch.cuda.current_stream().cuda_stream
