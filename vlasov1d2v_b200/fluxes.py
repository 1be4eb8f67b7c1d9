"""The semi-discrete DG right-hand side of the 1D2V Vlasov equation.

Mirrors ``DGFlux`` of crewsdw/Vlasov1D2V (``main/fluxes.py:13-207``).  The whole operator --
flux products, the three ``up`` contractions, the upwind face fluxes in x, u and v with the
lift, and the Jacobian-weighted sum -- is one native kernel launch (``vl_rhs``).
"""
from __future__ import annotations

import torch

from . import _device, _lib
from .context import get_context


class DGFlux:
    def __init__(self, resolutions, orders, flux_coefficients):
        # resolutions are ghost-inclusive (main/main.py:148-150)
        self.resolutions = resolutions
        self.orders = orders
        self.acceleration_coefficient = flux_coefficients
        self.grid_axis = (0, 2, 4)
        self.sub_element_axis = (1, 3, 5)

    def _ctx(self, f, elliptic, grids):
        if elliptic.magnetic_field is None:
            raise ValueError("set the magnetic field first (Elliptic.set_magnetic_field)")
        return get_context(grids, precision=_device.precision_of(f),
                           accel=self.acceleration_coefficient, bfield=elliptic.magnetic_field,
                           kappa=elliptic.poisson_coefficient)

    def _apply(self, function, elliptic, grids, weights):
        f = _device.as_tensor(function).contiguous()
        ctx = self._ctx(f, elliptic, grids)
        E = _device.as_tensor(elliptic.electric_field, dtype=torch.float64).contiguous()
        out = torch.zeros_like(f)
        if weights is None:
            ctx.rhs(f, E, out, xhalo=_lib.VL_XHALO_GHOST)
        else:
            ctx.rhs_weighted(f, E, out, weights, xhalo=_lib.VL_XHALO_GHOST)
        return _device.wrap(out)

    def semi_discrete_rhs(self, function, elliptic, basis, grids):
        """J_x F_x + J_u F_u + J_v F_v on the interior; ghost rows of the result are zero
        (the reference computes garbage there and its caller discards it)."""
        return self._apply(function, elliptic, grids, None)

    def x_flux(self, function, basis, grid_u, elliptic=None, grids=None):
        """F_x without the Jacobian (``main/fluxes.py:107-115``); needs ``grids`` and an
        ``elliptic`` for the native context."""
        return self._apply(function, elliptic, grids, (1.0, 0.0, 0.0))

    def u_flux(self, function, basis, elliptic, grid_v, grids=None):
        """F_u without the Jacobian (``main/fluxes.py:117-138``)."""
        return self._apply(function, elliptic, grids, (0.0, 1.0, 0.0))

    def v_flux(self, function, basis, elliptic, grid_u, grids=None):
        """F_v without the Jacobian (``main/fluxes.py:140-153``)."""
        return self._apply(function, elliptic, grids, (0.0, 0.0, 1.0))
