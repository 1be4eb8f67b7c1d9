"""ctypes binding of ``libvlasov1d2v.so`` (the C ABI in ``include/vlasov1d2v.h``).

The library is the only compute path: if it is missing or fails to load, every GPU entry
point raises.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("VLASOV1D2V_LIB") or os.path.join(HERE, "libvlasov1d2v.so")

VL_OK = 0
VL_FP64 = 0
VL_FP32 = 1
VL_XHALO_GHOST = 0
VL_XHALO_PERIODIC = 1
ABI_VERSION = 2

# every symbol include/vlasov1d2v.h declares (checked by the CPU test suite)
EXPORTED = (
    "vl_ctx_create", "vl_ctx_destroy", "vl_last_error", "vl_abi_version", "vl_state_elems",
    "vl_workspace_bytes", "vl_rhs", "vl_rhs_weighted", "vl_moment", "vl_poisson", "vl_field_energy", "vl_adapt_dt",
    "vl_rk_stage", "vl_run_state_init", "vl_ssp_rk3_steps", "vl_sync_ghosts",
    "vl_ssp_rk3_steps_noalloc", "vl_initial_state", "vl_smooth_edges", "vl_interpolate",
    "vl_set_background", "vl_set_background_pairs", "vl_ens_create", "vl_ens_destroy", "vl_ens_workspace_bytes", "vl_ens_bind",
    "vl_ens_schedule", "vl_ens_schedule_by_order", "vl_ens_commit", "vl_ens_steps", "vl_mlp_dims", "vl_mlp_forward",
    "vl_mlp_partial_floats", "vl_mlp_backward", "vl_mlp_adam", "vl_closure_features", "vl_closure_apply",
    "vl_poisson_dg", "vl_axpby_interior",
)
NOALLOC_SCRATCH_BYTES = 1 << 20
VL_CLOSURE_PLAIN = 0
VL_CLOSURE_CHARGE = 1
VL_ENS_NATIVE_AUTO = 0xFFFFFFFF

_c_dbl_p = ctypes.POINTER(ctypes.c_double)


class VlConfig(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_int32), ("precision", ctypes.c_int32),
        ("nx", ctypes.c_int32), ("nu", ctypes.c_int32), ("nv", ctypes.c_int32),
        ("n", ctypes.c_int32), ("n_modes", ctypes.c_int32), ("reserved0", ctypes.c_int32),
        ("accel", ctypes.c_double), ("bfield", ctypes.c_double), ("kappa", ctypes.c_double),
        ("jx", ctypes.c_double), ("ju", ctypes.c_double), ("jv", ctypes.c_double),
        ("dx", ctypes.c_double), ("du", ctypes.c_double), ("dv", ctypes.c_double),
        ("length_x", ctypes.c_double), ("umax", ctypes.c_double), ("vmax", ctypes.c_double),
        ("courant", ctypes.c_double),
        ("up", _c_dbl_p), ("xi", _c_dbl_p), ("xw", _c_dbl_p), ("u_nodes", _c_dbl_p),
        ("v_nodes", _c_dbl_p), ("wave_numbers", _c_dbl_p), ("dft_ell", _c_dbl_p),
        ("dft_phase", _c_dbl_p), ("dft_qnode", _c_dbl_p),
    ]


class VlRunState(ctypes.Structure):
    _fields_ = [
        ("dt", ctypes.c_double), ("dt_next", ctypes.c_double), ("time", ctypes.c_double),
        ("final_time", ctypes.c_double), ("steps", ctypes.c_int64), ("max_steps", ctypes.c_int64),
        ("active", ctypes.c_int32), ("active_next", ctypes.c_int32), ("status", ctypes.c_int32),
        ("hist_capacity", ctypes.c_int32), ("energy_hist", ctypes.c_void_p),
        ("time_hist", ctypes.c_void_p), ("dt_hist", ctypes.c_void_p),
        ("reserved", ctypes.c_double * 4),
    ]


RUN_STATE_BYTES = ctypes.sizeof(VlRunState)


class VlasovError(RuntimeError):
    """Raised when an entry point of the native library returns a non-zero status."""

    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} failed with status {code}: {msg}")
        self.code = code


_lock = threading.Lock()
_lib = None


def _declare(lib):
    vp = ctypes.c_void_p
    i = ctypes.c_int
    lib.vl_ctx_create.argtypes = [ctypes.POINTER(VlConfig), ctypes.POINTER(vp)]
    lib.vl_ctx_destroy.argtypes = [vp]
    lib.vl_last_error.restype = ctypes.c_char_p
    lib.vl_abi_version.restype = i
    lib.vl_state_elems.argtypes = [vp]
    lib.vl_state_elems.restype = ctypes.c_size_t
    lib.vl_workspace_bytes.argtypes = [vp]
    lib.vl_workspace_bytes.restype = ctypes.c_size_t
    lib.vl_rhs.argtypes = [vp, vp, vp, vp, i, vp]
    lib.vl_rhs_weighted.argtypes = [vp, vp, vp, vp, i, _c_dbl_p, vp]
    lib.vl_moment.argtypes = [vp, vp, vp, vp]
    lib.vl_poisson.argtypes = [vp, vp, vp, vp, vp]
    lib.vl_field_energy.argtypes = [vp, vp, vp, vp]
    lib.vl_adapt_dt.argtypes = [vp, vp, vp, vp]
    lib.vl_rk_stage.argtypes = [vp, i, vp, vp, vp, vp, vp, i, vp, vp]
    lib.vl_run_state_init.argtypes = [vp, vp, vp, ctypes.c_double, ctypes.c_int64, vp, vp, vp,
                                      ctypes.c_int32, vp, vp]
    lib.vl_ssp_rk3_steps.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i, vp]
    lib.vl_sync_ghosts.argtypes = [vp, vp, vp, vp]
    lib.vl_ssp_rk3_steps_noalloc.argtypes = [vp, vp, vp, vp, vp, vp, vp, i, vp]
    i32 = ctypes.c_int32
    lib.vl_set_background.argtypes = [vp, vp, vp]
    lib.vl_set_background_pairs.argtypes = [vp, vp]
    lib.vl_poisson_dg.argtypes = [vp, vp, vp, vp, vp, i32, vp, vp, vp]
    lib.vl_axpby_interior.argtypes = [vp, vp, vp, ctypes.c_double, ctypes.c_double, vp]
    lib.vl_ens_create.argtypes = [ctypes.POINTER(vp), i32, ctypes.POINTER(vp)]
    lib.vl_ens_destroy.argtypes = [vp]
    lib.vl_ens_workspace_bytes.argtypes = [vp, i32]
    lib.vl_ens_workspace_bytes.restype = ctypes.c_size_t
    lib.vl_ens_bind.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp]
    lib.vl_ens_schedule.argtypes = [vp, i32, i32, i32]
    lib.vl_ens_schedule_by_order.argtypes = [vp, i32, ctypes.c_uint32]
    lib.vl_ens_commit.argtypes = [vp]
    lib.vl_ens_steps.argtypes = [vp, i32, vp]
    f32, f64 = ctypes.c_float, ctypes.c_double
    pi32 = ctypes.POINTER(i32)
    lib.vl_mlp_dims.argtypes = [pi32, pi32, pi32, pi32, pi32]
    lib.vl_mlp_forward.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp, vp]
    lib.vl_mlp_partial_floats.argtypes = [i32]
    lib.vl_mlp_partial_floats.restype = ctypes.c_size_t
    lib.vl_mlp_backward.argtypes = [vp, vp, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    lib.vl_mlp_adam.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, f32, f32, f32, f32, i32, f32, vp]
    lib.vl_closure_features.argtypes = [vp, i32, i32, i32, i32, vp, f64, f64, vp, vp, f64, f64, f64, vp, vp, vp]
    lib.vl_closure_apply.argtypes = [vp, i32, i32, i32, i32, vp, vp, f64, f32, vp, f64, vp, i32, vp, vp]
    lib.vl_initial_state.argtypes = [vp, i32, i32, i32, i32, i32, vp, vp, vp, vp, vp, vp,
                                     ctypes.c_double, vp]
    lib.vl_smooth_edges.argtypes = [vp, i32, i32, i32, i32, i32, vp]
    lib.vl_interpolate.argtypes = [vp, i32, i32, i32, i32, i32, ctypes.POINTER(i32), vp, vp, vp,
                                   i32, i32, i32, vp, vp]
    for name in EXPORTED:
        if name not in ("vl_last_error", "vl_abi_version", "vl_state_elems", "vl_workspace_bytes",
                        "vl_ens_workspace_bytes", "vl_mlp_partial_floats"):
            getattr(lib, name).restype = i


def load(path: str | None = None):
    """Load (once) and return the native library.  Raises if it is missing."""
    global _lib
    with _lock:
        if _lib is not None and path is None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise FileNotFoundError(
                f"{p} is missing: build it with `python -m vlasov1d2v_b200.build` "
                "(this package has no CPU fallback)")
        lib = ctypes.CDLL(p)
        _declare(lib)
        if lib.vl_abi_version() != ABI_VERSION:
            raise RuntimeError("libvlasov1d2v ABI version mismatch")
        if path is None:
            _lib = lib
        return lib


def check(fn_name: str, code: int):
    if code != VL_OK:
        msg = load().vl_last_error()
        raise VlasovError(fn_name, code, msg.decode() if msg else "")


def call(fn_name: str, *args):
    lib = load()
    check(fn_name, getattr(lib, fn_name)(*args))
