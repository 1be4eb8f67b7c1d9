"""Set-up of the loss-cone cyclotron-harmonic problem, as the reference driver builds it.

``build`` reproduces the object graph of crewsdw/Vlasov1D2V's ``main/main.py:36-166``
(normalisation triplet, basis, grids over x in [-L/2, L/2) with L = 2 pi / (k / (omega_p /
omega_c)), velocities in +-8.5 v_t, loss-cone distribution, elliptic solver with the initial
field, flux operator and SSP-RK3 stepper) with the plotting and file output left out.
``cos_perturbed`` builds the benchmark initial states f0(u, v) (1 + a cos kx [+ noise]).
"""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import torch

from . import _device
from .basis import Basis3D
from .elliptic import Elliptic
from .fluxes import DGFlux
from .grid import Distribution, Grid3D
from .reference import Reference
from .timestep import Stepper

# normalisation triplet of the reference driver (main/main.py:38-43)
MP = 1.67262158e-27
C_LIGHT = 299792458.0
E_CHARGE = 1.602176634e-19
TRIPLET = np.array([1.0e21, (MP * C_LIGHT ** 2.0) / E_CHARGE, 1.0])
MASS_FRACTION = 1836.15267343


def default_reference():
    return Reference(triplet=TRIPLET, mass_fraction=MASS_FRACTION)


def loss_cone(grids, vt, ring_j):
    """Ring distribution on every node incl. ghosts (``main/grid.py:253-268``), host FP64."""
    d = Distribution(vt=vt, ring_j=ring_j, resolutions=[grids.x.res, grids.u.res, grids.v.res],
                     orders=[grids.x.order] * 3, perturbation=False)
    return d.initial_array(grids)


def cos_x_factor(grids, amp, noise=0.0, seed=0):
    """1 + amp cos(k1 x) + noise r(x) on the x nodes incl. ghosts, k1 the fundamental mode of
    the x domain and r uniform in [-1, 1] per interior x node (seeded; ghost x nodes take the
    periodic copy)."""
    k1 = 2.0 * np.pi / (grids.x.high - grids.x.low)
    mod = 1.0 + amp * np.cos(k1 * grids.x.arr)
    if noise:
        rng = np.random.default_rng(seed)
        r = rng.uniform(-1.0, 1.0, size=(grids.x.res, grids.x.order))
        rr = np.zeros_like(mod)
        rr[1:-1] = r
        rr[0] = r[-1]
        rr[-1] = r[0]
        mod = mod + noise * rr
    return mod


def cos_perturbed(grids, vt, ring_j, amp, noise=0.0, seed=0):
    """Host FP64 f0(u, v) (1 + amp cos(k1 x) + noise r(x)) (see ``cos_x_factor``)."""
    f0 = loss_cone(grids, vt, ring_j)
    return f0 * cos_x_factor(grids, amp, noise, seed)[:, :, None, None, None, None]


def build(res, order, *, om_pc=10.0, k=0.886, vmax=8.5, ring_j=6, perturbation="eigenmode",
          amp=1.0e-3, noise=0.0, seed=0, precision="fp64", final_time=2.0, write_time=0.1,
          om=-0.349j, batch_steps=32, verbose=False, background_split=True):
    """Build (refs, basis, grids, distribution, elliptic, flux, stepper) on the current device.

    ``perturbation``: ``"eigenmode"`` (the reference's Bessel-series mode with amplitude
    ``amp``, ``main/grid.py:201-242``), ``"cos"`` (f0 (1 + amp cos kx + noise r(x))) or
    ``None``.  The initial field is solved from n0 - mean(n0) as ``main/main.py:131`` does.
    """
    refs = default_reference()
    orders = np.array([order] * 3)
    basis = Basis3D(orders)
    k_est = k / om_pc
    L = 2.0 * np.pi / k_est
    lows = np.array([-L / 2.0, -vmax * refs.vt_e, -vmax * refs.vt_e])
    highs = np.array([L / 2.0, vmax * refs.vt_e, vmax * refs.vt_e])
    resolutions = np.array(res)
    grids = Grid3D(basis=basis, lows=lows, highs=highs, resolutions=resolutions)
    dist = Distribution(vt=refs.vt_e, ring_j=ring_j, resolutions=resolutions, orders=orders,
                        om=om, om_pc=om_pc, delta_n=amp, perturbation=(perturbation == "eigenmode"),
                        precision=precision, background_split=background_split)
    dist.initialize_quad_weights(grids)
    if perturbation == "cos":
        # loss cone times the x factor, formed on the device (vl_initial_state)
        dist.perturbation = False
        dist.initialize_gpu(grids, x_factor=cos_x_factor(grids, amp, noise=noise, seed=seed))
    else:
        dist.initialize_gpu(grids)
    el = Elliptic(poisson_coefficient=refs.charge_density_multiplier)
    el.set_magnetic_field(magnetic_field=(refs.omp_e_tau / refs.omc_e_tau) / om_pc)
    n0 = _device.plain(dist.moment_zero())
    el.poisson2(charge_density=n0 - torch.mean(n0), grid=grids.x, basis=basis.b1)
    flux = DGFlux(resolutions=resolutions + 2, orders=orders,
                  flux_coefficients=refs.electron_acceleration_multiplier)
    try:
        stepper = Stepper(time_order=3, space_order=order, write_time=write_time,
                          final_time=final_time, batch_steps=batch_steps, verbose=verbose)
    except IndexError:  # the Courant table stops at n = 9 (main/timestep.py:27)
        stepper = None
    return SimpleNamespace(refs=refs, basis=basis, grids=grids, f=dist, elliptic=el, flux=flux,
                           stepper=stepper, L=L, lows=lows, highs=highs, orders=orders,
                           resolutions=resolutions)


def dof(res, order):
    return int(res[0] * res[1] * res[2]) * order ** 3


__all__ = ["build", "cos_perturbed", "cos_x_factor", "loss_cone", "default_reference", "dof"]
