"""Nodal DG basis on Legendre-Gauss-Lobatto (LGL) points, orders 1..10.

Mirrors ``Basis1D`` / ``Basis3D`` of crewsdw/Vlasov1D2V (``main/basis.py:87-317``).  These are
host-side set-up tables (NumPy, FP64); the kernels receive them through the context.

Parity notes
  * LGL nodes/weights: closed forms for n <= 6 (the textbook expressions), and for n >= 7 the
    roots of P'_{n-1} computed by Newton iteration in 40-digit decimal arithmetic and rounded
    to double.  The reference hard-codes the same constants (``main/basis.py:9-57``).
  * Matrices that carry Legendre polynomial values are evaluated through the polynomials'
    power-series coefficients (``scipy.special.legendre``) in the reference's summation order,
    and entries below the reference's roundoff thresholds are zeroed
    (``main/basis.py:161, 186, 200``), so the tables match the reference to the last bit.
"""
from __future__ import annotations

from decimal import Decimal, getcontext

import numpy as np
import scipy.special as sp


def _lgl_decimal(n, digits=40):
    """Interior LGL nodes (roots of P'_{n-1}) and all weights via Decimal Newton iterations."""
    getcontext().prec = digits + 10
    m = n - 1

    def legendre_p_dp(x):
        p0, p1 = Decimal(1), x
        for k in range(1, m):
            p0, p1 = p1, ((2 * k + 1) * x * p1 - k * p0) / (k + 1)
        # P'_m from (x^2 - 1) P'_m = m (x P_m - P_{m-1})
        dp = m * (x * p1 - p0) / (x * x - 1)
        return p1, dp, p0

    def dp_ddp(x):
        p, dp, _ = legendre_p_dp(x)
        # (1 - x^2) P''_m = 2 x P'_m - m (m + 1) P_m
        ddp = (2 * x * dp - m * (m + 1) * p) / (1 - x * x)
        return dp, ddp

    guesses = np.cos(np.pi * (np.arange(1, m) + 0.25) / (m + 0.5))[::-1]
    roots = []
    for g in guesses:
        x = Decimal(repr(float(g)))
        for _ in range(60):
            dp, ddp = dp_ddp(x)
            step = dp / ddp
            x -= step
            if abs(step) < Decimal(10) ** (-digits):
                break
        roots.append(x)
    roots.sort()
    weights = []
    for x in [Decimal(-1)] + roots + [Decimal(1)]:
        p, _, _ = legendre_p_dp(x) if abs(x) != 1 else (Decimal(1) if x > 0 else Decimal((-1) ** m), 0, 0)
        weights.append(Decimal(2) / (Decimal(n * m) * p * p))
    return [float(r) for r in roots], [float(w) for w in weights]


def lgl_nodes(n):
    if n == 1:
        return [0]
    if n == 2:
        return [-1, 1]
    if n == 3:
        return [-1, 0, 1]
    if n == 4:
        a = np.sqrt(1 / 5)
        return [-1, -a, a, 1]
    if n == 5:
        a = np.sqrt(3 / 7)
        return [-1, -a, 0, a, 1]
    if n == 6:
        a = np.sqrt(1 / 3 + 2 * np.sqrt(7) / 21)
        b = np.sqrt(1 / 3 - 2 * np.sqrt(7) / 21)
        return [-1, -a, -b, b, a, 1]
    roots, _ = _lgl_decimal(n)
    half = [abs(r) for r in roots[: (n - 2) // 2]]
    mid = [0.0] if (n - 2) % 2 == 1 else []
    inner = [-h for h in half] + mid + half[::-1]
    return [-1] + inner + [1]


def lgl_weights(n):
    if n == 1:
        return [2]
    if n == 2:
        return [1, 1]
    if n == 3:
        return [1 / 3, 4 / 3, 1 / 3]
    if n == 4:
        return [1 / 6, 5 / 6, 5 / 6, 1 / 6]
    if n == 5:
        return [1 / 10, 49 / 90, 32 / 45, 49 / 90, 1 / 10]
    if n == 6:
        a = (14 - np.sqrt(7)) / 30
        b = (14 + np.sqrt(7)) / 30
        return [1 / 15, a, b, b, a, 1 / 15]
    _, w = _lgl_decimal(n)
    half = w[: (n + 1) // 2]
    return half + half[: n // 2][::-1]


class Basis1D:
    """LGL nodal basis of one dimension (``main/basis.py:87-116``)."""

    def __init__(self, order):
        self.order = int(order)
        if not 1 <= self.order <= 10:
            raise ValueError("order must be in 1..10")
        self.nodes = lgl_nodes(self.order)
        self.weights = lgl_weights(self.order)
        self.eigenvalues = self.set_eigenvalues()
        self.vandermonde_inverse = self.set_vandermonde_inverse()
        self.mass = self.mass_matrix()
        self.invm = self.inv_mass_matrix()
        self.face_mass = np.eye(self.order)[:, np.array([0, -1])]
        self.adv = self.advection_matrix()
        self.stf = self.adv.T
        self.np_up = self.internal_flux()
        self.np_xi = self.invm[:, np.array([0, -1])].copy()
        self.der = self.derivative_matrix()
        self._dev = {}

    # -- device copies (torch tensors on the current CUDA device), created on first use --
    def _device(self, name, arr):
        import torch

        dev = torch.cuda.current_device()
        key = (name, dev)
        if key not in self._dev:
            self._dev[key] = torch.as_tensor(arr, dtype=torch.float64, device=f"cuda:{dev}")
        return self._dev[key]

    @property
    def up(self):
        return self._device("up", self.np_up)

    @property
    def xi(self):
        return self._device("xi", self.np_xi)

    @property
    def d_mass(self):
        return self._device("mass", self.mass)

    # -- tables ---------------------------------------------------------------------------------
    def set_eigenvalues(self):
        ev = np.array([(2.0 * s + 1) / 2.0 for s in range(self.order - 1)])
        return np.append(ev, (self.order - 1) / 2.0)

    def set_vandermonde_inverse(self):
        n = self.order
        polys = [sp.legendre(s) for s in range(n)]
        return np.array([[self.weights[j] * self.eigenvalues[s] * polys[s](self.nodes[j])
                          for j in range(n)] for s in range(n)])

    def mass_matrix(self):
        n = self.order
        p = sp.legendre(n - 1)
        v = np.multiply(self.weights, p(self.nodes))
        a = -n * (n - 1) / (2 * (2 * n - 1))
        return np.diag(self.weights) + a * np.outer(v, v)

    def inv_mass_matrix(self):
        n = self.order
        v = sp.legendre(n - 1)(self.nodes)
        return np.diag(np.divide(1.0, self.weights)) + (n / 2) * np.outer(v, v)

    def _pairwise(self, coef, outer_poly_at_i, inner_poly_at_j, weight_index):
        n = self.order
        polys = [sp.legendre(s) for s in range(n)]
        derivs = [p.deriv() for p in polys]
        out = np.zeros((n, n))
        for i in range(n):
            for j in range(n):
                acc = 0
                for s in range(n):
                    pi = (derivs[s] if outer_poly_at_i == "d" else polys[s])(self.nodes[i])
                    pj = (derivs[s] if inner_poly_at_j == "d" else polys[s])(self.nodes[j])
                    acc = acc + coef(s) * pi * pj
                w = self.weights[j] if weight_index == "j" else self.weights[i] * self.weights[j]
                out[i, j] = w * acc
        return out

    def advection_matrix(self):
        adv = self._pairwise(lambda s: self.eigenvalues[s], "p", "d", "ij")
        adv[np.abs(adv) < 1.0e-15] = 0
        return adv

    def internal_flux(self):
        up = self._pairwise(lambda s: (2 * s + 1) / 2, "p", "d", "j")
        up[np.abs(up) < 1.0e-10] = 0
        return up

    def derivative_matrix(self):
        der = self._pairwise(lambda s: self.eigenvalues[s], "d", "p", "j")
        der[np.abs(der) < 1.0e-15] = 0
        return der

    def fourier_factors(self, midpoints, J, wave_numbers):
        """The two factors of the high-order DFT tensor (``main/basis.py:204-228``): the exact
        Fourier transform of the nodal basis, ell[j, m] (spherical Bessel functions of each
        Legendre mode combined with the inverse Vandermonde matrix), and the element phases
        exp(-i k_m mid_e).  Host complex128, [n][M] and [nx][M]."""
        signs = np.sign(wave_numbers)
        signs[np.where(wave_numbers == 0)] = 1.0
        p_tilde = np.array([(signs ** s) * np.exp(-1j * np.pi / 2.0 * s) *
                            sp.spherical_jn(s, np.absolute(wave_numbers) / J)
                            for s in range(self.order)])
        ell_tilde = np.matmul(self.vandermonde_inverse.T, p_tilde)
        phase = np.exp(-1j * np.tensordot(midpoints, wave_numbers, axes=0))
        return ell_tilde, phase

    def fourier_transform_array(self, midpoints, J, wave_numbers):
        """High-order DFT tensor T[e, j, m] = phase[e, m] ell[j, m] (``main/basis.py:204-228``),
        host complex128."""
        ell_tilde, phase = self.fourier_factors(midpoints, J, wave_numbers)
        transform = np.multiply(phase[:, :, None], ell_tilde.T)
        return np.ascontiguousarray(np.transpose(transform, (0, 2, 1)))

    def interpolate_values(self, grid, arr):
        """Values of the nodal polynomial on the grid's fine points (``main/basis.py:230-250``)."""
        xi = grid.J * (grid.arr_fine[1:-1, :] - grid.midpoints[:, None])
        ps = np.array([sp.legendre(s)(xi) for s in range(self.order)])
        ell = np.transpose(np.tensordot(self.vandermonde_inverse, ps, axes=([0], [0])), [1, 0, 2])
        return np.multiply(ell, np.asarray(arr)[:, :, None]).sum(axis=1)


class Basis3D:
    """Tensor product of three 1D bases (``main/basis.py:283-289``)."""

    def __init__(self, orders):
        self.orders = orders
        self.b1 = Basis1D(orders[0])
        self.b2 = Basis1D(orders[1])
        self.b3 = Basis1D(orders[2])

    @staticmethod
    def _fine_lagrange(basis, grid, lim):
        """ell[e][i][p]: the element's Lagrange polynomials at its fine points, for the elements
        lim[0] <= e < lim[1] (ghost-inclusive indices), as ``main/basis.py:296-309`` builds
        them (Legendre series through the inverse Vandermonde matrix).  Host FP64."""
        xi = grid.J * (grid.arr_fine[lim[0]:lim[1], :] - grid.midpoints[lim[0] - 1:lim[1] - 1, None])
        ps = np.array([sp.legendre(s)(xi) for s in range(basis.order)])
        return np.ascontiguousarray(
            np.transpose(np.tensordot(basis.vandermonde_inverse, ps, axes=([0], [0])), [1, 0, 2]))

    def interpolate_values(self, grids, arr, limits):
        """Values of the nodal state on the fine points of the elements in ``limits``
        (``main/basis.py:291-317``): device kernel ``vl_interpolate``; returns a device array
        [ex, fx, eu, fu, ev, fv] (FP64).  ``grids`` needs fine points in all three directions
        (``Grid3D(..., fine_all=True)``)."""
        import ctypes

        import torch

        from . import _device, _lib

        t = _device.as_tensor(arr)
        if t.dim() != 6:
            raise ValueError("arr must be the 6-D state f[X, n, U, n, V, n]")
        t = t.contiguous()
        X, n, U, _, V, _ = t.shape
        lims = [int(v) for pair in limits for v in pair]
        ells = [self._fine_lagrange(b, g, lim) for b, g, lim in
                ((self.b1, grids.x, limits[0]), (self.b2, grids.u, limits[1]), (self.b3, grids.v, limits[2]))]
        dev = [torch.as_tensor(e, device=t.device) for e in ells]
        fx, fu, fv = (e.shape[2] for e in ells)
        ex, eu, ev = (lims[1] - lims[0], lims[3] - lims[2], lims[5] - lims[4])
        out = torch.empty((ex, fx, eu, fu, ev, fv), dtype=torch.float64, device=t.device)
        c_lims = (ctypes.c_int32 * 6)(*lims)
        _lib.call("vl_interpolate", t.data_ptr(), _lib.VL_FP64 if t.dtype == torch.float64 else _lib.VL_FP32,
                  X - 2, U - 2, V - 2, n, c_lims, dev[0].data_ptr(), dev[1].data_ptr(),
                  dev[2].data_ptr(), fx, fu, fv, out.data_ptr(), _device.stream_handle())
        return _device.wrap(out)

    def interpolate_values_host(self, grids, arr, limits):
        """Host NumPy form of ``interpolate_values`` (the reference's own expression)."""
        ell_x, ell_u, ell_v = (self._fine_lagrange(b, g, lim) for b, g, lim in
                               ((self.b1, grids.x, limits[0]), (self.b2, grids.u, limits[1]),
                                (self.b3, grids.v, limits[2])))
        x_lim, u_lim, v_lim = limits
        arr_r = np.asarray(arr)[x_lim[0]:x_lim[1], :, u_lim[0]:u_lim[1], :, v_lim[0]:v_lim[1], :]
        values = np.multiply(ell_x[:, :, :, None, None, None, None], arr_r[:, :, None, :, :, :, :]).sum(axis=1)
        values = np.multiply(ell_u[None, None, :, :, :, None, None], values[:, :, :, :, None, :, :]).sum(axis=3)
        values = np.multiply(ell_v[None, None, None, None, :, :, :], values[:, :, :, :, :, :, None]).sum(axis=5)
        return values
