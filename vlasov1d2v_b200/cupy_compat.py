"""A ``cupy`` stand-in over this package's CUDA tensors, for drivers written against CuPy.

The reference driver (``main/main.py``) and the reference's own loop call a handful of CuPy
functions on the arrays the solver classes return: ``cp.asnumpy`` on flattened states
(``main/main.py:87-88``, ``:171``, ``:215``), ``cp.asarray(n0) - cp.mean(n0)`` for the initial
field (``main/main.py:131``), ``cp.amax(cp.absolute(...))`` for the speeds
(``main/timestep.py:237``).  Installing this module as ``sys.modules["cupy"]`` lets such a driver
run unchanged on ``vlasov1d2v_b200``: device arrays are ``CudaArray`` tensors (with CuPy's
``.get()``), host arrays stay NumPy.  It is an adapter for the driver's glue code, not a
compute path: the solver's work runs in the native library.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _device

ndarray = _device.CudaArray
pi = np.pi
inf = np.inf
float64 = np.float64
float32 = np.float32


def _t(x):
    """A CUDA tensor for any array-like (device tensors pass through)."""
    return _device.as_tensor(x)


def asarray(a, dtype=None):
    if isinstance(a, torch.Tensor):
        t = _device.plain(a)
        if t.device.type != "cuda":
            t = t.to(_device.device())
    else:
        arr = np.asarray(a)
        t = torch.as_tensor(np.ascontiguousarray(arr), device=_device.device())
    if dtype is not None:
        t = t.to(torch.float32 if np.dtype(dtype) == np.float32 else torch.float64)
    return _device.wrap(t)


array = asarray


def asnumpy(a):
    if isinstance(a, torch.Tensor):
        return _device.plain(a).detach().cpu().numpy()
    return np.asarray(a)


def _red(fn, a, axis=None):
    t = _t(a)
    if axis is None:
        return _device.wrap(fn(t))
    return _device.wrap(fn(t, dim=axis))


def mean(a, axis=None):
    return _red(torch.mean, a, axis)


def sum(a, axis=None):  # noqa: A001  (CuPy's name)
    return _red(torch.sum, a, axis)


def amax(a, axis=None):
    if axis is None:
        return _device.wrap(torch.max(_t(a)))
    return _device.wrap(torch.amax(_t(a), dim=axis))


def amin(a, axis=None):
    if axis is None:
        return _device.wrap(torch.min(_t(a)))
    return _device.wrap(torch.amin(_t(a), dim=axis))


max = amax  # noqa: A001
min = amin  # noqa: A001


def absolute(a):
    return _device.wrap(torch.abs(_t(a)))


abs = absolute  # noqa: A001


def sqrt(a):
    return _device.wrap(torch.sqrt(_t(a)))


def exp(a):
    return _device.wrap(torch.exp(_t(a)))


def sin(a):
    return _device.wrap(torch.sin(_t(a)))


def cos(a):
    return _device.wrap(torch.cos(_t(a)))


def isnan(a):
    return _device.wrap(torch.isnan(_t(a)))


def zeros(shape, dtype=np.float64):
    return asarray(np.zeros(shape, dtype=dtype))


def zeros_like(a):
    return _device.wrap(torch.zeros_like(_t(a)))


def ones_like(a):
    return _device.wrap(torch.ones_like(_t(a)))


def copy(a):
    return _device.wrap(_t(a).clone())


def where(condition=None, x=None, y=None):
    return _device.wrap(torch.where(_t(condition).bool(), _t(x), _t(y)))


class random:  # noqa: N801  (CuPy's namespace)
    """``cupy.random.seed / rand / randn`` (FP64 device arrays from torch's generator)."""

    @staticmethod
    def seed(s):
        torch.cuda.manual_seed(int(s))

    @staticmethod
    def rand(*shape):
        return _device.wrap(torch.rand(shape, dtype=torch.float64, device=_device.device()))

    @staticmethod
    def randn(*shape):
        return _device.wrap(torch.randn(shape, dtype=torch.float64, device=_device.device()))


class cuda:  # noqa: N801  (CuPy's namespace)
    """``cupy.cuda.Stream.null.synchronize()`` as the reference's commented timing code uses."""

    class Stream:
        class null:  # noqa: N801
            @staticmethod
            def synchronize():
                torch.cuda.synchronize()


def install():
    """Make ``import cupy`` resolve to this module (returns the module)."""
    import sys

    mod = sys.modules[__name__]
    sys.modules["cupy"] = mod
    return mod
