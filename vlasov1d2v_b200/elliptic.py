"""Field solves: the spectral (high-order DFT) Poisson solve and the field energy.

Mirrors ``Elliptic`` of crewsdw/Vlasov1D2V (``main/elliptic.py``).  ``poisson2`` and
``electric_energy`` run as native kernels; ``build_central_flux_operator`` / ``invert`` /
``poisson`` (the DG central-flux solve, used by the reference only at set-up and by its
unused linear stepper) are kept with the same signatures, built on the host and applied with
device tensor algebra.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _device
from .context import get_context


class Elliptic:
    def __init__(self, poisson_coefficient):
        self.central_flux_operator = None
        self.gradient_operator = None
        self.inv_op = None
        self.potential = None
        self.electric_field = None
        self.magnetic_field = None
        self.poisson_coefficient = poisson_coefficient

    # -- DG central-flux operator (main/elliptic.py:24-83), host set-up ----------------------------
    def build_central_flux_operator(self, grid, basis):
        """The bordered central-flux Laplacian (host) and the DG gradient map (device) of
        ``central_flux_matrices``."""
        bordered, grad_src = central_flux_matrices(grid, basis)
        self.central_flux_operator = bordered
        self.gradient_operator = _device.wrap(torch.as_tensor(grad_src, device=_device.device()))

    def invert(self):
        self.inv_op = _device.wrap(torch.as_tensor(np.linalg.inv(self.central_flux_operator),
                                                   device=_device.device()))

    def poisson(self, charge_density, grid, basis, anti_alias=True):
        """DG central-flux Poisson solve (``main/elliptic.py:85-115``): one native kernel
        (``vl_poisson_dg``) over the operator tables of ``build_central_flux_operator`` /
        ``invert``."""
        import ctypes

        from . import _lib

        if self.inv_op is None or self.gradient_operator is None:
            raise RuntimeError("call build_central_flux_operator(grid, basis) and invert() first")
        rho = _device.as_tensor(charge_density).contiguous()
        ctx = get_context(grid, kappa=self.poisson_coefficient)
        E = torch.empty((grid.res_ghosts, grid.order), dtype=torch.float64, device=rho.device)
        phi = torch.empty((grid.res, grid.order), dtype=torch.float64, device=rho.device)
        mass = _device.plain(basis.d_mass).contiguous()
        _lib.call("vl_poisson_dg", ctx.handle, ctypes.c_void_p(rho.data_ptr()),
                  ctypes.c_void_p(_device.plain(self.inv_op).data_ptr()), ctypes.c_void_p(mass.data_ptr()),
                  ctypes.c_void_p(_device.plain(self.gradient_operator).data_ptr()), int(bool(anti_alias)),
                  ctypes.c_void_p(E.data_ptr()), ctypes.c_void_p(phi.data_ptr()),
                  ctypes.c_void_p(_device.stream_handle()))
        self.potential = _device.wrap(phi)
        self.electric_field = _device.wrap(E)

    # -- hot path ------------------------------------------------------------------------------------
    def poisson2(self, charge_density, grid, basis=None):
        """Spectral Poisson solve in high-order-DFT coefficients (``main/elliptic.py:117-145``),
        one native kernel: forward DFT, -c/(i k) and -c/k^2 with the k = 0 mode dropped, inverse
        DFT at the LGL nodes, periodic ghost rows."""
        ctx = get_context(grid, kappa=self.poisson_coefficient)
        charge = _device.as_tensor(charge_density, dtype=torch.float64).contiguous()
        E = torch.empty((grid.res_ghosts, grid.order), dtype=torch.float64, device=charge.device)
        phi = torch.empty((grid.res, grid.order), dtype=torch.float64, device=charge.device)
        ctx.poisson(charge, E, phi)
        self.electric_field = _device.wrap(E)
        self.potential = _device.wrap(phi)

    def set_magnetic_field(self, magnetic_field):
        self.magnetic_field = magnetic_field

    def electric_energy(self, grid):
        """0.5 sum w E^2 over the interior nodes (``main/elliptic.py:150-151``); a 0-d device
        array (``.get()`` returns the host value)."""
        ctx = get_context(grid, kappa=self.poisson_coefficient)
        E = _device.as_tensor(self.electric_field, dtype=torch.float64).contiguous()
        out = torch.empty(1, dtype=torch.float64, device=E.device)
        ctx.field_energy(E, out)
        return _device.wrap(out[0])


def central_flux_matrices(grid, basis):
    """Bordered matrix of the DG central-flux Laplacian and the DG gradient map, host FP64.

    Both are assembled directly as linear maps on the nodal vector q (length res n, element
    major): with J0 q = q[e, 0] - q[e-1, n-1] and J1 q = q[e, n-1] - q[e+1, 0] the trace jumps at
    the left and right face of every element (periodic), the gradient is
    g = (I kron der) q + xi_L (J0 q) / 2 - xi_R (J1 q) / 2, and the operator is
    (I kron stf) g + e_0 (J0 g / 2 + J0 q) + e_{n-1} (-J1 g / 2 + J1 q)
    (face_mass selects the first and last node of each element).  The reference stores each map
    with the source node first (row = source, column = destination), so both are returned in
    that convention: the Laplacian bordered by the quadrature weights (zero-mean gauge row and
    column) with entries below 1e-15 cleared, as ``main/elliptic.py:73-78`` does, and the
    gradient as [i, j, e, k] = node (e, k) of the gradient of the unit vector at (i, j)."""
    res, n = grid.res, grid.order
    N = res * n
    eye = np.eye(res)
    nxt = np.roll(eye, 1, axis=1)    # (nxt x)[e] = x[e+1]
    prv = np.roll(eye, -1, axis=1)   # (prv x)[e] = x[e-1]
    first = np.kron(eye, np.eye(n)[:1])   # res x N: q[e, 0]
    last = np.kron(eye, np.eye(n)[-1:])   # res x N: q[e, n-1]
    jump_left = first - prv @ last
    jump_right = last - nxt @ first
    xi = basis.np_xi
    lift_left = np.kron(eye, xi[:, :1])   # N x res: xi[:, 0] into element e
    lift_right = np.kron(eye, xi[:, 1:])
    grad = np.kron(eye, basis.der) + 0.5 * (lift_left @ jump_left) - 0.5 * (lift_right @ jump_right)
    lap = (np.kron(eye, basis.stf) @ grad + first.T @ (0.5 * (jump_left @ grad) + jump_left) +
           last.T @ (-0.5 * (jump_right @ grad) + jump_right))
    qw = np.asarray(grid.np_quad_weights, dtype=np.float64).reshape(N)
    bordered = np.zeros((N + 1, N + 1))
    bordered[:N, :N] = lap.T
    bordered[:N, N] = qw
    bordered[N, :N] = qw
    bordered[np.abs(bordered) < 1.0e-15] = 0
    return bordered, np.ascontiguousarray(grad.T.reshape(res, n, res, n))
