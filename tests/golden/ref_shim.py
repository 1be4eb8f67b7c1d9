"""Import shim that runs the reference's CuPy modules on the CPU with NumPy.

Test infrastructure only: it is used by ``make_golden.py`` (fixture generation) and by the
CPU tests that cross-check the oracle against the reference when the reference checkout is
present in the container.  Nothing on the product path imports it.

What the shim provides (each item is something the reference's hot-path modules call):

* ``cupy`` -> a NumPy-backed module whose arrays are an ``ndarray`` subclass with ``.get()``
  (``main/timestep.py:85``, ``main/timestep.py:102``, ``main/timestep.py:238``).
* keyword ``where(condition=, x=, y=)`` (``main/grid.py:35-36``, ``main/fluxes.py:185-186``).
* CuPy's complex division by zero (``nan+nanj``), which ``main/elliptic.py:124-128`` relies on
  to zero the k = 0 Fourier mode through ``nan_to_num``.  NumPy would give ``inf`` there.
* ``np.math`` (removed in NumPy 2; used at ``main/grid.py:213`` and ``main/grid.py:253``).
* stub ``matplotlib.pyplot`` (imported at module level by ``basis.py``, ``grid.py``,
  ``fluxes.py``).
"""
import math
import os
import sys
import types

import numpy as np

# the reference checkout's ``main/`` directory; there is no default: the variable must name it
REFERENCE_MAIN = os.environ.get("VLASOV_REFERENCE_MAIN", "")


class CpArray(np.ndarray):
    """ndarray with CuPy's ``.get()`` (device -> host copy, here a plain view)."""

    def get(self):
        return np.asarray(self)

    def __array_wrap__(self, arr, context=None, return_scalar=False):
        # keep 0-d results as arrays so ``.get()`` stays available (CuPy never returns
        # Python scalars from array expressions)
        return np.asarray(arr).view(CpArray)


def _wrap(x):
    if isinstance(x, np.ndarray):
        return x.view(CpArray)
    if isinstance(x, (np.floating, np.complexfloating, np.integer, np.bool_)):
        return np.asarray(x).view(CpArray)
    return x


def _wrapped(fn):
    def inner(*args, **kwargs):
        return _wrap(fn(*args, **kwargs))

    inner.__name__ = getattr(fn, "__name__", "fn")
    return inner


def _where(condition=None, x=None, y=None, *args):
    if args or (condition is not None and x is None and y is None):
        return _wrap(np.where(condition, *args))
    return _wrap(np.where(condition, x, y))


def _divide(a, b, *args, **kwargs):
    a_arr = np.asarray(a)
    b_arr = np.asarray(b)
    with np.errstate(divide="ignore", invalid="ignore"):
        out = np.divide(a_arr, b_arr, *args, **kwargs)
    if np.iscomplexobj(out):
        zero = np.broadcast_to(b_arr == 0, out.shape)
        if np.any(zero):
            out = np.array(out, copy=True)
            out[zero] = complex(np.nan, np.nan)
    return _wrap(out)


def _asarray(a, dtype=None):
    return np.asarray(a, dtype=dtype).view(CpArray)


def _asnumpy(a):
    return np.asarray(a)


def _make_cupy():
    cp = types.ModuleType("cupy")
    for name in ("tensordot", "transpose", "multiply", "roll", "zeros", "nan_to_num", "real",
                 "zeros_like", "copy", "amax", "absolute", "mean", "ones", "exp", "sqrt",
                 "ascontiguousarray", "array", "matmul", "sum", "cos", "sin", "arange",
                 "linspace", "ones_like", "isnan", "abs", "max", "min", "amin", "reshape",
                 "conj", "imag"):
        setattr(cp, name, _wrapped(getattr(np, name)))
    cp.where = _where
    cp.divide = _divide
    cp.asarray = _asarray
    cp.asnumpy = _asnumpy
    cp.ndarray = CpArray
    cp.pi = np.pi
    cp.inf = np.inf
    return cp


def _make_matplotlib():
    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")

    def _noop(*args, **kwargs):
        return None

    for name in ("figure", "plot", "show", "imshow", "colorbar", "title", "grid", "xlabel",
                 "ylabel", "legend", "tight_layout", "contourf", "semilogy", "axis", "savefig"):
        setattr(plt, name, _noop)
    mpl.pyplot = plt
    mpl.rc = _noop
    return mpl, plt


def install():
    """Install the shims and put the reference's ``main/`` directory on ``sys.path``.

    Returns the imported reference modules as a namespace (basis, grid, elliptic, fluxes,
    timestep, reference).
    """
    if not REFERENCE_MAIN:
        raise RuntimeError("set VLASOV_REFERENCE_MAIN to the reference checkout's main/ directory")
    if not os.path.isdir(REFERENCE_MAIN):
        raise FileNotFoundError(REFERENCE_MAIN)
    if not hasattr(np, "math"):
        np.math = math
    sys.modules["cupy"] = _make_cupy()
    mpl, plt = _make_matplotlib()
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", plt)
    if REFERENCE_MAIN not in sys.path:
        sys.path.insert(0, REFERENCE_MAIN)
    import basis as ref_basis  # noqa: E402
    import elliptic as ref_elliptic  # noqa: E402
    import fluxes as ref_fluxes  # noqa: E402
    import grid as ref_grid  # noqa: E402
    import reference as ref_reference  # noqa: E402
    import timestep as ref_timestep  # noqa: E402

    return types.SimpleNamespace(basis=ref_basis, grid=ref_grid, elliptic=ref_elliptic,
                                 fluxes=ref_fluxes, timestep=ref_timestep,
                                 reference=ref_reference)


def available():
    return bool(REFERENCE_MAIN) and os.path.isdir(REFERENCE_MAIN)
