"""Grids, the high-order-DFT tables and the phase-space distribution.

Mirrors ``Grid1D``, ``Grid3D`` and ``Distribution`` of crewsdw/Vlasov1D2V (``main/grid.py``).
Coordinates and spectral tables are built on the host exactly as the reference builds them
(same NumPy expressions and order), then handed to the native context.  The distribution
``.arr`` is a CUDA tensor in the reference's ghost-inclusive layout
``[X, n, U, n, V, n]`` (``main/grid.py:262-268``); FP64 by default, FP32 for the mixed-precision
form.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.special as sp

from . import _device
from .context import get_context


class Grid1D:
    """One axis with ghost elements (``main/grid.py:10-88``)."""

    def __init__(self, low, high, res, basis, spectrum=False, fine=False):
        self.low = low
        self.high = high
        self.res = int(res)
        self.res_ghosts = int(res + 2)
        self.order = basis.order
        self.basis = basis
        self.length = self.high - self.low
        self.dx = self.length / self.res
        self.J = 2.0 / self.dx
        self.np_quad_weights = np.tensordot(np.ones(self.res), np.asarray(basis.weights, dtype=float),
                                            axes=0)
        self.arr = np.zeros((self.res_ghosts, self.order))
        self.create_grid(basis.nodes)
        self.midpoints = np.array([(self.arr[i, -1] + self.arr[i, 0]) / 2.0
                                   for i in range(1, self.res_ghosts - 1)])
        self.arr_max = np.amax(abs(self.arr))
        self.np_one_negatives = np.where(self.arr < 0, 1, 0)
        self.np_one_positives = np.where(self.arr >= 0, 1, 0)
        if fine:
            fine_num = 25
            self.arr_fine = np.array([np.linspace(self.arr[i, 0], self.arr[i, -1], num=fine_num)
                                      for i in range(self.res_ghosts)])
        self.spectrum = bool(spectrum)
        if spectrum:
            self.nyquist_number = 2.5 * self.length // self.dx
            self.k1 = 2.0 * np.pi / self.length
            self.wave_numbers = self.k1 * np.arange(1 - self.nyquist_number, self.nyquist_number)
            self.np_grid_phases = np.exp(1j * np.tensordot(self.wave_numbers, self.arr[1:-1, :], axes=0))
            self.np_spectral_transform = basis.fourier_transform_array(self.midpoints, self.J,
                                                                       self.wave_numbers)
            # the factors the native field solve uses: T[e, j, m] = phase[e, m] ell[j, m] and
            # exp(i k_m x_{e,j}) = conj(phase[e, m]) qnode[j, m]
            ell, phase = basis.fourier_factors(self.midpoints, self.J, self.wave_numbers)
            self.np_dft_ell = np.ascontiguousarray(ell)
            self.np_dft_phase = np.ascontiguousarray(phase)
            self.np_dft_qnode = np.ascontiguousarray(
                np.exp(1j * np.multiply.outer(self.arr[1] - self.midpoints[0], self.wave_numbers)))
        self._vl_cache = {}

    def create_grid(self, nodes):
        """Ghost-inclusive node coordinates (``main/grid.py:55-70``)."""
        min_gs = self.low - self.dx
        max_gs = self.high
        nodes = (np.array(nodes) + 1) / 2
        xl = np.linspace(min_gs, max_gs, num=self.res_ghosts)
        for i in range(self.res_ghosts):
            self.arr[i, :] = xl[i] + self.dx * nodes

    # -- device views (CuPy arrays in the reference) --------------------------------------------
    @property
    def arr_cp(self):
        return _device.const(self, "arr", self.arr)

    @property
    def quad_weights(self):
        return _device.const(self, "quad_weights", self.np_quad_weights)

    @property
    def one_negatives(self):
        return _device.const(self, "one_negatives", self.np_one_negatives)

    @property
    def one_positives(self):
        return _device.const(self, "one_positives", self.np_one_positives)

    @property
    def d_wave_numbers(self):
        return _device.const(self, "wave_numbers", self.wave_numbers)

    @property
    def grid_phases(self):
        return _device.const(self, "grid_phases", self.np_grid_phases, complex_=True)

    @property
    def spectral_transform(self):
        return _device.const(self, "spectral_transform", self.np_spectral_transform, complex_=True)

    def fourier_basis(self, function):
        """Fourier coefficients of a grid function (``main/grid.py:78-82``)."""
        import torch

        f = _device.as_tensor(function).to(torch.complex128)
        c = torch.tensordot(f, self.spectral_transform, dims=([0, 1], [0, 1]))
        return _device.wrap(c * self.dx / self.length)

    def sum_fourier(self, coefficients):
        """Re-sum Fourier coefficients at the nodes (``main/grid.py:84-88``)."""
        import torch

        c = _device.as_tensor(coefficients).to(torch.complex128)
        return _device.wrap(torch.real(torch.tensordot(c, self.grid_phases, dims=([0], [0]))))


class Grid3D:
    """x, u, v axes (``main/grid.py:91-109``)."""

    def __init__(self, basis, lows, highs, resolutions, fine_x=False, fine_all=False):
        fx = bool(fine_x or fine_all)
        self.x = Grid1D(low=lows[0], high=highs[0], res=resolutions[0], basis=basis.b1, spectrum=True,
                        fine=fx)
        self.u = Grid1D(low=lows[1], high=highs[1], res=resolutions[1], basis=basis.b2, fine=fine_all)
        self.v = Grid1D(low=lows[2], high=highs[2], res=resolutions[2], basis=basis.b3, fine=fine_all)
        self.no_ghost_slice = (slice(1, self.x.res_ghosts - 1), slice(self.x.order),
                               slice(1, self.u.res_ghosts - 1), slice(self.u.order),
                               slice(1, self.v.res_ghosts - 1), slice(self.v.order))
        self._vl_cache = {}


def smooth_edges(arr):
    """Average each element-face node with its neighbour's (``main/grid.py:116-134``), in
    place on the device (``vl_smooth_edges``: six passes in the reference's order).  Returns
    the device array (a host array is copied to the device first)."""
    import torch

    from . import _lib

    t = _device.as_tensor(arr)
    if t.dim() != 6 or not t.is_contiguous():
        raise ValueError("arr must be a contiguous 6-D state f[X, n, U, n, V, n]")
    X, n, U, _, V, _ = t.shape
    _lib.call("vl_smooth_edges", t.data_ptr(), _lib.VL_FP64 if t.dtype == torch.float64 else _lib.VL_FP32,
              X - 2, U - 2, V - 2, n, _device.stream_handle())
    return _device.wrap(t)


class Distribution:
    """Phase-space distribution f[X, n, U, n, V, n] (``main/grid.py:137-321``).

    ``precision`` selects the state type: ``"fp64"`` (the reference's, default) or ``"fp32"``
    (mixed precision: FP32 state and contractions; FP64 moment, Poisson and energy).

    ``background_split`` (FP32 only, default on): ``arr`` holds delta f = f - f0(u, v) with
    f0 an x-independent FP64 background (the loss cone of the initial state, or the x-average of
    a state given to ``set_array``).  The FP32 x derivative then acts on the O(perturbation)
    part only instead of cancelling the O(1) background; the stage kernels add the FP64-built
    RHS of f0.  ``full_array()`` returns f = f0 + delta f; ``moment_zero()`` the full density.
    """

    def __init__(self, vt, ring_j, resolutions, orders, perturbation=True, om=0.9, om_pc=1.0,
                 delta_n=0.01, precision="fp64", background_split=True):
        self.ring_j = ring_j
        self.vt = vt
        self.om = om
        self.om_pc = om_pc
        self.delta_n = delta_n
        self.arr = None
        self.arr_explicit_copy = None
        self.arr_next = None
        self.perturbation = perturbation
        self.x_res, self.u_res, self.v_res = int(resolutions[0]), int(resolutions[1]), int(resolutions[2])
        self.x_ord, self.u_ord, self.v_ord = int(orders[0]), int(orders[1]), int(orders[2])
        self.quad_weights = None
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision must be 'fp64' or 'fp32'")
        self.precision = precision
        self.background_split = bool(background_split) and precision == "fp32"
        self.background = None      # host FP64 f0[U, n, V, n] when split
        self._bg_cache = {}
        self._grids = None

    @property
    def dtype(self):
        import torch

        return torch.float64 if self.precision == "fp64" else torch.float32

    @property
    def shape(self):
        return (self.x_res + 2, self.x_ord, self.u_res + 2, self.u_ord, self.v_res + 2, self.v_ord)

    def set_array(self, arr):
        """Install a host or device array as the state (cast to this distribution's precision).
        With the background split, ``arr`` is the full f: its x-average (interior x nodes)
        becomes the background f0 and the state holds f - f0."""
        import torch

        if self.background_split:
            t = _device.as_tensor(arr, dtype=torch.float64)
            if tuple(t.shape) != self.shape:
                raise ValueError(f"state shape {tuple(t.shape)} != {self.shape}")
            f0 = t[1:-1].mean(dim=(0, 1))
            self._set_background(f0.cpu().numpy())
            self.arr = _device.wrap((t - f0).to(self.dtype).contiguous())
            return
        t = _device.as_tensor(arr, dtype=self.dtype)
        if tuple(t.shape) != self.shape:
            raise ValueError(f"state shape {tuple(t.shape)} != {self.shape}")
        self.arr = _device.wrap(t.contiguous())

    def _set_background(self, f0):
        self.background = np.ascontiguousarray(f0, dtype=np.float64)
        self._bg_cache = {}

    def full_array(self):
        """The full state f (FP64 device array): f0 + delta f with the split, else ``arr``."""
        import torch

        t = _device.plain(self.arr)
        if not self.background_split or self.background is None:
            return _device.wrap(t)
        f0 = torch.as_tensor(self.background, device=t.device)
        return _device.wrap(t.double() + f0)

    def background_tables(self, grids, accel, bfield):
        """RHS tables of the background f0 for ``vl_set_background`` (host FP64 arithmetic,
        stored float32 on the device), cached per (accel, B).  Velocity-slab layout
        [U, n, V, n]; ghost entries zero.  f0 is continuous across element faces, so the u
        derivative with the upwind lift of either side agrees (to rounding); the v direction's
        upwind side depends on u only and is folded in."""
        import torch

        key = (float(accel), float(bfield))
        if key in self._bg_cache:
            return self._bg_cache[key]
        f0 = self.background
        n = self.u_ord
        up = np.asarray(grids.u.basis.np_up, dtype=np.float64)
        xi = np.asarray(grids.u.basis.np_xi, dtype=np.float64)
        # u direction: contraction over j (axis 1) of f0[a, m, b, k]
        cu = np.einsum("jm,ambk->ajbk", up, f0)
        du = np.zeros_like(f0)
        du[1:-1] = (cu[1:-1] + xi[None, :, 0, None, None] * f0[:-2, n - 1][:, None]
                    - xi[None, :, 1, None, None] * f0[1:-1, n - 1][:, None])
        # v direction: contraction over k (axis 3), upwind side from sv = -a B u
        cv = np.einsum("km,ajbm->ajbk", up, f0)
        sv = accel * (-bfield * grids.u.arr)                     # [U, n]
        pos = (sv >= 0.0)[:, :, None, None]
        left_p = xi[None, None, None, :, 0] * f0[:, :, :-2, n - 1][..., None] - xi[None, None, None, :, 1] * f0[:, :, 1:-1, n - 1][..., None]
        left_m = xi[None, None, None, :, 0] * f0[:, :, 1:-1, 0][..., None] - xi[None, None, None, :, 1] * f0[:, :, 2:, 0][..., None]
        dv = np.zeros_like(f0)
        dv[:, :, 1:-1] = cv[:, :, 1:-1] + np.where(pos, left_p, left_m)
        ju, jv = grids.u.J, grids.v.J
        vv = grids.v.arr[None, None, :, :]                       # [1, 1, V, n]
        rv = jv * sv[:, :, None, None] * dv
        tabs = {"rb": ju * accel * bfield * vv * du + rv, "eu": ju * accel * du}
        for t in tabs.values():   # only interior elements are read
            t[0] = t[-1] = 0.0
            t[:, :, 0] = t[:, :, -1] = 0.0
        dev = _device.device()
        out = {k: torch.as_tensor(np.ascontiguousarray(v), dtype=torch.float32, device=dev)
               for k, v in tabs.items()}
        rows, cols = f0.shape[0] * f0.shape[1], f0.shape[2] * f0.shape[3]
        if cols % 2 == 0:   # both tables interleaved per column pair (vl_set_background_pairs)
            eu2 = out["eu"].reshape(rows, cols // 2, 2)
            rb2 = out["rb"].reshape(rows, cols // 2, 2)
            out["pairs"] = torch.cat([eu2, rb2], dim=2).contiguous()
        self._bg_cache[key] = out
        return out

    def initialize_next(self):
        import torch

        self.arr_next = _device.wrap(torch.zeros_like(self.arr))

    def reset_array(self, grids):
        self.arr[grids.no_ghost_slice] = self.arr_next[grids.no_ghost_slice]

    def swap_ghost_cells_of_array(self):
        self.arr[0] = self.arr[-2].clone()
        self.arr[-1] = self.arr[1].clone()

    def swap_ghost_cells_of_copy(self):
        self.arr_explicit_copy[0] = self.arr_explicit_copy[-2].clone()
        self.arr_explicit_copy[-1] = self.arr_explicit_copy[1].clone()

    def copy_for_explicit_advance(self):
        self.arr_explicit_copy = _device.wrap(self.arr.clone())

    # -- initial condition (host NumPy, then uploaded) ------------------------------------------
    def eigenfunction(self, grids):
        """Bessel-series eigenmode perturbation (``main/grid.py:201-242``), host complex128."""
        u = np.tensordot(grids.u.arr, np.ones_like(grids.v.arr), axes=0)
        v = np.tensordot(np.ones_like(grids.u.arr), grids.v.arr, axes=0)
        r = np.sqrt(u ** 2.0 + v ** 2.0)
        phi = np.arctan2(v, u)
        beta = - grids.x.k1 * r * self.om_pc
        x = 0.5 * (r / self.vt) ** 2.0
        f0 = 1 / (2.0 * np.pi * (self.vt ** 2.0) * math.factorial(self.ring_j)) * np.multiply(
            x ** self.ring_j, np.exp(-x))
        df_dv = np.multiply(f0, (self.ring_j / (x + 1.0e-16) - 1.0)) / (self.vt ** 2.0)
        terms_n = 20
        upsilon = np.array([n / (n - self.om) * np.multiply(sp.jv(n, beta), np.exp(-1j * n * phi))
                            for n in range(-terms_n, terms_n + 1)]).sum(axis=0)
        eig = 0 + 0j
        eig += np.multiply(df_dv, upsilon) / grids.x.k1 ** 2.0
        vel_mode = -1j * np.multiply(np.exp(1j * np.multiply(beta, np.sin(phi))), eig)
        return 2.0 * self.delta_n * np.real(np.tensordot(np.exp(1j * grids.x.k1 * grids.x.arr),
                                                         vel_mode, axes=0))

    def initial_array(self, grids):
        """Loss-cone ring f0 on every node incl. ghosts (``main/grid.py:244-279``), host FP64."""
        factor = 1.0 / ((2.0 ** self.ring_j) * (2.0 * np.pi) * (self.vt ** 2.0) *
                        math.factorial(self.ring_j))
        ix = np.tensordot(np.ones(grids.x.res_ghosts), np.ones(grids.x.order), axes=0)
        iu = np.tensordot(np.ones(grids.u.res_ghosts), np.ones(grids.u.order), axes=0)
        iv = np.tensordot(np.ones(grids.v.res_ghosts), np.ones(grids.v.order), axes=0)
        rsq = (np.tensordot(grids.u.arr ** 2.0, iv, axes=0) +
               np.tensordot(iu, grids.v.arr ** 2.0, axes=0)) / (self.vt ** 2.0)
        rad_j = rsq ** self.ring_j
        gauss = np.exp(-0.5 * rsq)
        pol_eig = np.multiply(rad_j, gauss)
        arr = factor * np.tensordot(ix, pol_eig, axes=0)
        if self.perturbation:
            arr = arr + self.eigenfunction(grids=grids)
        return arr

    def velocity_tables(self, grids):
        """The O(velocity) parts of the initial state, host FP64: the loss-cone values
        factor * rsq^j exp(-rsq/2) on the velocity nodes [U, n, V, n] (``main/grid.py:253-268``)
        and, with a perturbation, the eigenmode's velocity part [U, n, V, n] (complex)."""
        factor = 1.0 / ((2.0 ** self.ring_j) * (2.0 * np.pi) * (self.vt ** 2.0) *
                        math.factorial(self.ring_j))
        iu = np.tensordot(np.ones(grids.u.res_ghosts), np.ones(grids.u.order), axes=0)
        iv = np.tensordot(np.ones(grids.v.res_ghosts), np.ones(grids.v.order), axes=0)
        rsq = (np.tensordot(grids.u.arr ** 2.0, iv, axes=0) +
               np.tensordot(iu, grids.v.arr ** 2.0, axes=0)) / (self.vt ** 2.0)
        pol = factor * np.multiply(rsq ** self.ring_j, np.exp(-0.5 * rsq))
        mode = None
        if self.perturbation:
            u = np.tensordot(grids.u.arr, np.ones_like(grids.v.arr), axes=0)
            v = np.tensordot(np.ones_like(grids.u.arr), grids.v.arr, axes=0)
            r = np.sqrt(u ** 2.0 + v ** 2.0)
            phi = np.arctan2(v, u)
            beta = - grids.x.k1 * r * self.om_pc
            x = 0.5 * (r / self.vt) ** 2.0
            f0 = 1 / (2.0 * np.pi * (self.vt ** 2.0) * math.factorial(self.ring_j)) * np.multiply(
                x ** self.ring_j, np.exp(-x))
            df_dv = np.multiply(f0, (self.ring_j / (x + 1.0e-16) - 1.0)) / (self.vt ** 2.0)
            upsilon = np.array([n / (n - self.om) * np.multiply(sp.jv(n, beta), np.exp(-1j * n * phi))
                                for n in range(-20, 21)]).sum(axis=0)
            eig = np.multiply(df_dv, upsilon) / grids.x.k1 ** 2.0
            mode = -1j * np.multiply(np.exp(1j * np.multiply(beta, np.sin(phi))), eig)
        return pol, mode

    def initialize_gpu(self, grids, x_factor=None):
        """Build the initial state on the device (``vl_initial_state``): the O(DOF) tensor
        product pol(u, v) [* x_factor(x)] [+ 2 delta_n Re(exp(i k1 x) mode(u, v))] is formed by
        the kernel from the host's O(velocity) tables."""
        import torch

        from . import _lib

        self._grids = grids
        pol, mode = self.velocity_tables(grids)
        dev = _device.device()
        f = torch.empty(self.shape, dtype=self.dtype, device=dev)
        keep = [torch.as_tensor(np.ascontiguousarray(pol), device=dev)]
        ptr = lambda a: a.data_ptr() if a is not None else None
        mx = None
        if x_factor is not None:
            mx = torch.as_tensor(np.ascontiguousarray(x_factor, dtype=np.float64), device=dev)
        cx = sx = vre = vim = None
        if mode is not None:
            ph = np.exp(1j * grids.x.k1 * grids.x.arr)
            cx = torch.as_tensor(np.ascontiguousarray(ph.real), device=dev)
            sx = torch.as_tensor(np.ascontiguousarray(ph.imag), device=dev)
            vre = torch.as_tensor(np.ascontiguousarray(mode.real), device=dev)
            vim = torch.as_tensor(np.ascontiguousarray(mode.imag), device=dev)
        if self.background_split:
            # the state is delta f = f - pol: the loss cone becomes the background
            self._set_background(pol)
            mx_host = (np.zeros(grids.x.arr.shape) if x_factor is None
                       else np.asarray(x_factor, dtype=np.float64) - 1.0)
            mx = torch.as_tensor(np.ascontiguousarray(mx_host), device=dev)
        _lib.call("vl_initial_state", f.data_ptr(),
                  _lib.VL_FP64 if self.precision == "fp64" else _lib.VL_FP32,
                  self.x_res, self.u_res, self.v_res, self.x_ord,
                  keep[0].data_ptr(), ptr(mx), ptr(cx), ptr(sx), ptr(vre), ptr(vim),
                  2.0 * self.delta_n, _device.stream_handle())
        torch.cuda.current_stream().synchronize()   # the host tables are freed on return
        self.arr = _device.wrap(f)

    def grid_order_gpu(self):
        self.arr = _device.wrap(self.arr.permute(0, 2, 4, 1, 3, 5).contiguous())

    def tensor_product_order_gpu(self):
        self.arr = _device.wrap(self.arr.permute(0, 3, 1, 4, 2, 5).contiguous())

    def grid_flatten_gpu(self):
        return _device.wrap(self.arr.reshape((self.x_res + 2) * self.x_ord,
                                             (self.u_res + 2) * self.u_ord,
                                             (self.v_res + 2) * self.v_ord))

    # -- moments (native kernel) -------------------------------------------------------------------
    def initialize_quad_weights(self, grids):
        """Velocity quadrature weights w_u w_v / (J_u J_v) (``main/grid.py:297-301``)."""
        import torch

        self._grids = grids
        qw = np.tensordot(grids.u.np_quad_weights, grids.v.np_quad_weights, axes=0) / (grids.u.J * grids.v.J)
        self.quad_weights = _device.wrap(torch.as_tensor(qw, device=_device.device()))

    def moment_zero(self):
        """Zeroth velocity moment over the interior (``main/grid.py:303-312``)."""
        return self.moment_zero_of_arr(self.arr)

    def moment_zero_of_copy(self):
        return self.moment_zero_of_arr(self.arr_explicit_copy)

    def moment_zero_of_arr(self, arr):
        import torch

        if self._grids is None:
            raise RuntimeError("call initialize_quad_weights(grids) or initialize_gpu(grids) first")
        t = _device.as_tensor(arr)
        ctx = get_context(self._grids, precision=_device.precision_of(t))
        rho = torch.empty((self.x_res, self.x_ord), dtype=torch.float64, device=t.device)
        ctx.moment(t, rho)
        if self.background_split and self.background is not None and t.data_ptr() == _device.plain(self.arr).data_ptr():
            # + the density of the background (x-independent, FP64 on the host)
            g = self._grids
            qw = np.tensordot(g.u.np_quad_weights, g.v.np_quad_weights, axes=0) / (g.u.J * g.v.J)
            rho0 = float(np.sum(self.background[1:-1, :, 1:-1, :] * qw))
            rho = rho + rho0
        return _device.wrap(rho)
