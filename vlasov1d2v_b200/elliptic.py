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
        res, order = grid.res, grid.order
        indicator = np.zeros((res, order))
        face_diff0 = np.zeros((res, 2))
        face_diff1 = np.zeros((res, 2))
        num_flux = np.zeros_like(face_diff0)
        grad_num_flux = np.zeros_like(face_diff1)
        op = np.zeros((res, order, res, order))
        grad_op = np.zeros_like(op)
        for i in range(res):
            for j in range(order):
                indicator[i, j] = 1.0
                face_diff0[:, 0] = indicator[:, 0] - np.roll(indicator[:, -1], 1)
                face_diff0[:, 1] = indicator[:, -1] - np.roll(indicator[:, 0], -1)
                num_flux[:, 0] = 0.5 * face_diff0[:, 0]
                num_flux[:, 1] = -0.5 * face_diff0[:, 1]
                grad = (np.tensordot(basis.der, indicator, axes=([1], [1])) +
                        np.tensordot(basis.np_xi, num_flux, axes=([1], [1]))).T
                face_diff1[:, 0] = grad[:, 0] - np.roll(grad[:, -1], 1)
                face_diff1[:, 1] = grad[:, -1] - np.roll(grad[:, 0], -1)
                grad_num_flux[:, 0] = 0.5 * face_diff1[:, 0]
                grad_num_flux[:, 1] = -0.5 * face_diff1[:, 1]
                operator = (np.tensordot(basis.stf, grad, axes=([1], [1])) +
                            np.tensordot(basis.face_mass, grad_num_flux + face_diff0, axes=([1], [1]))).T
                op[i, j, :, :] = operator
                grad_op[i, j, :, :] = grad
                indicator[i, j] = 0
        qw = grid.np_quad_weights
        op0 = np.hstack([op.reshape(res * order, res * order), qw.reshape(res * order, 1)])
        self.central_flux_operator = np.vstack([op0, np.append(qw.flatten(), 0)])
        self.central_flux_operator[np.abs(self.central_flux_operator) < 1.0e-15] = 0
        self.gradient_operator = _device.wrap(torch.as_tensor(grad_op, device=_device.device()))

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
