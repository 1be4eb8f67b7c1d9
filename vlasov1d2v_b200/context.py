"""Native context: one ``vl_ctx`` of the C library per problem set-up.

A context is created from the grids (x with its DFT tables, u, v), the basis matrices and the
physics scalars (acceleration multiplier, B, Poisson coefficient, Courant number) and the state
precision, and is cached on the grid object (``get_context``).  Its methods are thin wrappers of
the C ABI (``include/vlasov1d2v.h``) on CUDA tensors, issued on torch's current stream.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._device import device, stream_handle

_XONLY_NODES = np.zeros(3)  # node coordinates of the one-element dummy u/v axes of an x-only context


def _dptr(arr):
    return np.ascontiguousarray(arr, dtype=np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class NativeContext:
    """Owns one ``vl_ctx`` (coefficient tables on the device) and a workspace buffer."""

    def __init__(self, *, x, u=None, v=None, precision="fp64", accel=0.0, bfield=0.0, kappa=0.0,
                 courant=1.0):
        lib = _lib.load()
        n = x.order
        if u is not None and (u.order != n or v.order != n):
            raise NotImplementedError("the kernels take the same LGL order in x, u and v")
        if not getattr(x, "spectrum", False):
            raise ValueError("the x grid needs its spectral tables (Grid1D(..., spectrum=True))")
        self.n = n
        self.nx = x.res
        self.nu = u.res if u is not None else 1
        self.nv = v.res if v is not None else 1
        self.precision = precision
        self.dtype = torch.float64 if precision == "fp64" else torch.float32
        self.accel, self.bfield, self.kappa, self.courant = accel, bfield, kappa, courant
        basis = x.basis
        unodes = u.arr if u is not None else np.zeros((3, n))
        vnodes = v.arr if v is not None else np.zeros((3, n))
        self._keep = []  # host arrays alive during vl_ctx_create

        def keep(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            self._keep.append(a)
            return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

        ell = np.ascontiguousarray(x.np_dft_ell, dtype=np.complex128)
        phase = np.ascontiguousarray(x.np_dft_phase, dtype=np.complex128)
        qnode = np.ascontiguousarray(x.np_dft_qnode, dtype=np.complex128)
        cfg = _lib.VlConfig()
        cfg.abi_version = _lib.ABI_VERSION
        cfg.precision = _lib.VL_FP64 if precision == "fp64" else _lib.VL_FP32
        cfg.nx, cfg.nu, cfg.nv, cfg.n = self.nx, self.nu, self.nv, n
        cfg.n_modes = int(len(x.wave_numbers))
        cfg.accel = float(accel)
        cfg.bfield = float(bfield)
        cfg.kappa = float(kappa)
        cfg.jx = float(x.J)
        cfg.ju = float(u.J) if u is not None else 1.0
        cfg.jv = float(v.J) if v is not None else 1.0
        cfg.dx = float(x.dx)
        cfg.du = float(u.dx) if u is not None else 1.0
        cfg.dv = float(v.dx) if v is not None else 1.0
        cfg.length_x = float(x.length)
        cfg.umax = float(u.arr_max) if u is not None else 0.0
        cfg.vmax = float(v.arr_max) if v is not None else 0.0
        cfg.courant = float(courant)
        cfg.up = keep(basis.np_up)
        cfg.xi = keep(basis.np_xi)
        cfg.xw = keep(np.asarray(basis.weights, dtype=np.float64))
        cfg.u_nodes = keep(unodes)
        cfg.v_nodes = keep(vnodes)
        cfg.wave_numbers = keep(x.wave_numbers)
        cfg.dft_ell = keep(ell.view(np.float64))
        cfg.dft_phase = keep(phase.view(np.float64))
        cfg.dft_qnode = keep(qnode.view(np.float64))
        self.device = device()
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check("vl_ctx_create", lib.vl_ctx_create(ctypes.byref(cfg), ctypes.byref(handle)))
        self._keep = []
        self.handle = handle
        self._lib = lib
        self.state_elems = int(lib.vl_state_elems(handle))
        self.workspace_bytes = int(lib.vl_workspace_bytes(handle))
        self._workspace = None
        self.state_shape = (self.nx + 2, n, self.nu + 2, n, self.nv + 2, n)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._lib.vl_ctx_destroy(h)
            except Exception:
                pass
            self.handle = None

    # ---------------------------------------------------------------------------------------
    @property
    def workspace(self):
        if self._workspace is None:
            self._workspace = torch.empty(max(self.workspace_bytes, 256), dtype=torch.uint8,
                                          device=self.device)
        return self._workspace

    def _check_state(self, t, name="state"):
        if t.dtype != self.dtype:
            raise TypeError(f"{name} dtype {t.dtype} != context precision {self.dtype}")
        if tuple(t.shape) != self.state_shape:
            raise ValueError(f"{name} shape {tuple(t.shape)} != {self.state_shape}")
        if not t.is_contiguous() or t.device != self.device:
            raise ValueError(f"{name} must be a contiguous tensor on {self.device}")

    def _check_field(self, t, shape, name):
        if t.dtype != torch.float64 or tuple(t.shape) != tuple(shape) or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous float64 tensor of shape {shape}")

    def rhs(self, f, E, out, xhalo=_lib.VL_XHALO_GHOST):
        self._check_state(f, "f")
        self._check_state(out, "out")
        self._check_field(E, (self.nx + 2, self.n), "E")
        _lib.call("vl_rhs", self.handle, _ptr(f), _ptr(E), _ptr(out), int(xhalo),
                  ctypes.c_void_p(stream_handle()))

    def rhs_weighted(self, f, E, out, weights, xhalo=_lib.VL_XHALO_GHOST):
        self._check_state(f, "f")
        self._check_state(out, "out")
        self._check_field(E, (self.nx + 2, self.n), "E")
        w = (ctypes.c_double * 3)(*[float(x) for x in weights])
        _lib.call("vl_rhs_weighted", self.handle, _ptr(f), _ptr(E), _ptr(out), int(xhalo),
                  ctypes.cast(w, ctypes.POINTER(ctypes.c_double)), ctypes.c_void_p(stream_handle()))

    def moment(self, f, rho):
        self._check_state(f, "f")
        self._check_field(rho, (self.nx, self.n), "rho")
        _lib.call("vl_moment", self.handle, _ptr(f), _ptr(rho), ctypes.c_void_p(stream_handle()))

    def poisson(self, charge, E, phi=None):
        self._check_field(charge, (self.nx, self.n), "charge_density")
        self._check_field(E, (self.nx + 2, self.n), "E")
        if phi is not None:
            self._check_field(phi, (self.nx, self.n), "phi")
        _lib.call("vl_poisson", self.handle, _ptr(charge), _ptr(E), _ptr(phi),
                  ctypes.c_void_p(stream_handle()))

    def field_energy(self, E, out):
        self._check_field(E, (self.nx + 2, self.n), "E")
        _lib.call("vl_field_energy", self.handle, _ptr(E), _ptr(out), ctypes.c_void_p(stream_handle()))

    def adapt_dt(self, E, out):
        self._check_field(E, (self.nx + 2, self.n), "E")
        _lib.call("vl_adapt_dt", self.handle, _ptr(E), _ptr(out), ctypes.c_void_p(stream_handle()))

    def rk_stage(self, stage, inp, fn, out, E, dt, xhalo=_lib.VL_XHALO_PERIODIC, partials=None):
        self._check_state(inp, "in")
        self._check_state(out, "out")
        if fn is not None:
            self._check_state(fn, "fn")
        _lib.call("vl_rk_stage", self.handle, int(stage), _ptr(inp), _ptr(fn), _ptr(out), _ptr(E),
                  _ptr(dt), int(xhalo), _ptr(partials), ctypes.c_void_p(stream_handle()))

    def set_background(self, tables):
        """Install (tables = dict rb, eu of float32 device tensors) or clear (None) the
        background-split RHS tables of the FP32 mixed form."""
        self._bg = tables   # keep the tensors alive while the context refers to them
        if tables is None:
            _lib.call("vl_set_background", self.handle, None, None)
        else:
            _lib.call("vl_set_background", self.handle, _ptr(tables["rb"]), _ptr(tables["eu"]))
            pairs = tables.get("pairs")
            _lib.call("vl_set_background_pairs", self.handle, None if pairs is None else _ptr(pairs))

    def sync_ghosts(self, f, stage):
        self._check_state(f, "f")
        if stage is not None:
            self._check_state(stage, "stage")
        _lib.call("vl_sync_ghosts", self.handle, _ptr(f), _ptr(stage), ctypes.c_void_p(stream_handle()))

    def run_state_init(self, state, E0, final_time, max_steps, energy_hist, time_hist, dt_hist,
                       energy0=None):
        cap = int(energy_hist.numel())
        _lib.call("vl_run_state_init", self.handle, _ptr(state), _ptr(E0), float(final_time),
                  int(max_steps), _ptr(energy_hist), _ptr(time_hist), _ptr(dt_hist), cap,
                  _ptr(energy0), ctypes.c_void_p(stream_handle()))

    def ssp_rk3_steps(self, f, sa, sb, E, phi, state, nsteps):
        self._check_state(f, "f")
        self._check_state(sa, "stage_a")
        self._check_state(sb, "stage_b")
        _lib.call("vl_ssp_rk3_steps", self.handle, _ptr(f), _ptr(sa), _ptr(sb), _ptr(E), _ptr(phi),
                  _ptr(state), _ptr(self.workspace), int(nsteps), ctypes.c_void_p(stream_handle()))


    def ssp_rk3_steps_noalloc(self, f, sa, sb, E, phi, state, nsteps):
        """The loop without a workspace argument: its scratch is a fixed device array inside
        the library (see ``vl_ssp_rk3_steps_noalloc`` in include/vlasov1d2v.h)."""
        self._check_state(f, "f")
        self._check_state(sa, "stage_a")
        self._check_state(sb, "stage_b")
        _lib.call("vl_ssp_rk3_steps_noalloc", self.handle, _ptr(f), _ptr(sa), _ptr(sb), _ptr(E),
                  _ptr(phi), _ptr(state), int(nsteps), ctypes.c_void_p(stream_handle()))


def get_context(grids, *, precision="fp64", accel=0.0, bfield=0.0, kappa=0.0, courant=1.0):
    """Cached context for a ``Grid3D`` (full phase space) or an x ``Grid1D`` (field-only)."""
    key = (precision, float(accel), float(bfield), float(kappa), float(courant),
           torch.cuda.current_device())
    cache = grids.__dict__.setdefault("_vl_cache", {})
    ctx = cache.get(key)
    if ctx is None:
        if hasattr(grids, "x"):
            ctx = NativeContext(x=grids.x, u=grids.u, v=grids.v, precision=precision, accel=accel,
                                bfield=bfield, kappa=kappa, courant=courant)
        else:
            ctx = NativeContext(x=grids, precision=precision, accel=accel, bfield=bfield,
                                kappa=kappa, courant=courant)
        cache[key] = ctx
    return ctx
