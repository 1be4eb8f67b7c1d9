"""CPU oracle for the 1D2V DG Vlasov-Poisson hot path (NumPy, FP64).

TEST INFRASTRUCTURE ONLY.  This module is the oracle: ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline / reference arms of ``bench.py`` may import it.  The product package
(``vlasov1d2v_b200``) never imports it and has no CPU fallback.

It restates, in NumPy, the algorithm of crewsdw/Vlasov1D2V's hot path:

* DG basis matrices (``main/basis.py:87-202``): LGL nodes/weights, inverse Vandermonde,
  inverse mass matrix, ``up`` (internal flux) and ``xi`` (lift) with the reference's roundoff
  cleaning (``main/basis.py:186``).
* Grids (``main/grid.py:10-109``): ghost-inclusive node coordinates, Jacobians, the
  high-order-DFT tensors (``main/grid.py:45-53``, ``main/basis.py:204-228``).
* The semi-discrete RHS (``main/fluxes.py:59-207``): flux products, ``up`` contraction,
  upwind faces with periodic ``roll`` over the ghost-inclusive element axis, lift.
* Zeroth velocity moment (``main/grid.py:297-321``).
* Spectral Poisson solve ``poisson2`` (``main/elliptic.py:117-145``) with CuPy's
  complex-division-by-zero behaviour (k = 0 mode -> nan -> 0), field energy
  (``main/elliptic.py:150-151``).
* Nonlinear SSP-RK3 (``main/timestep.py:141-187``), adaptive dt (``main/timestep.py:231-242``),
  the main loop's bookkeeping (``main/timestep.py:81-103``).

Parity is pinned by ``tests/test_oracle_golden.py`` against fixtures generated from the
reference itself (``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
from numpy.polynomial import legendre as npleg
from scipy import special as sp

# ----------------------------------------------------------------------------------------------
# normalisation (main/reference.py:13-63)
# ----------------------------------------------------------------------------------------------
_ME = 9.10938188e-31
_MP = 1.67262158e-27
_E = 1.60217646e-19
_EPS0 = 8.854187e-12
_MU0 = 4.0e-7 * np.pi
_C = 1.0 / np.sqrt(_EPS0 * _MU0)


@dataclass
class Normalisation:
    """Dimensionless coefficients derived from a (density, temperature, Te/Ti) triplet."""

    vt_e: float
    accel: float  # electron acceleration multiplier (main/reference.py:61)
    kappa: float  # charge-density multiplier (main/reference.py:63)
    omp_e_tau: float
    omc_e_tau: float


def normalisation(triplet, mass_fraction) -> Normalisation:
    n, T, TeTi = float(triplet[0]), float(triplet[1]), float(triplet[2])
    Ld = np.sqrt(_EPS0 * T * TeTi / (n * _E))
    p = _E * n * T
    B = np.sqrt(p * _MU0)
    v = B / np.sqrt(_MU0 * _MP * n)
    tau = Ld / v
    omp_p = tau * np.sqrt(_E * _E * n / (_EPS0 * _MP))
    omp_e = tau * np.sqrt(_E * _E * n / (_EPS0 * _ME * mass_fraction))
    omc_e = tau * _E * B / (_ME * mass_fraction)
    dp = _C * tau / omp_p
    ae = mass_fraction * _ME / _MP
    Te = TeTi * T
    vt_e = np.sqrt(_E * Te / (_ME * mass_fraction)) / v
    length = (vt_e * v) / (omp_e / tau)
    accel = (-1.0 / ae) * (length / dp)
    kappa = -omp_p ** 2.0 * (dp / length)
    return Normalisation(vt_e=vt_e, accel=accel, kappa=kappa, omp_e_tau=omp_e, omc_e_tau=omc_e)


def default_normalisation() -> Normalisation:
    """The triplet of the reference driver (``main/main.py:39-43``)."""
    mp = 1.67262158e-27
    c = 299792458.0
    e = 1.602176634e-19
    return normalisation(np.array([1.0e21, (mp * c ** 2.0) / e, 1.0]), 1836.15267343)


# ----------------------------------------------------------------------------------------------
# basis (main/basis.py:87-228)
# ----------------------------------------------------------------------------------------------
def lgl_nodes_weights(n):
    """LGL nodes and weights.  Interior nodes are the roots of P'_{n-1}; they are polished by
    Newton iterations carried out in extended precision (``np.longdouble``) on the Legendre
    three-term recurrence and then rounded to float64.  Weights are 2 / (n (n-1) P_{n-1}^2).
    (The reference hard-codes the same constants to ~22 digits, ``main/basis.py:9-57``.)"""
    if n == 1:
        return np.array([0.0]), np.array([2.0])
    if n == 2:
        return np.array([-1.0, 1.0]), np.array([1.0, 1.0])
    ld = np.longdouble
    c = np.zeros(n)
    c[n - 1] = 1.0
    guess = np.sort(npleg.legroots(npleg.legder(c)).real).astype(ld)

    def p_dp_ddp(x):
        # P_{m}, P'_{m}, P''_{m} at x for m = n - 1 by the recurrence
        p0, p1 = np.ones_like(x), x.copy()
        d0, d1 = np.zeros_like(x), np.ones_like(x)
        e0, e1 = np.zeros_like(x), np.zeros_like(x)
        for k in range(1, n - 1):
            kk = ld(k)
            p2 = ((2 * kk + 1) * x * p1 - kk * p0) / (kk + 1)
            d2 = ((2 * kk + 1) * (p1 + x * d1) - kk * d0) / (kk + 1)
            e2 = ((2 * kk + 1) * (2 * d1 + x * e1) - kk * e0) / (kk + 1)
            p0, p1, d0, d1, e0, e1 = p1, p2, d1, d2, e1, e2
        return p1, d1, e1

    x = guess
    for _ in range(8):
        _, d, e = p_dp_ddp(x)
        x = x - d / e
    x = (x - x[::-1]) / 2
    if (n - 2) % 2 == 1:
        x[(n - 2) // 2] = 0
    pn, _, _ = p_dp_ddp(x)
    w = ld(2) / (ld(n) * ld(n - 1) * pn * pn)
    nodes = np.concatenate([[-1.0], x.astype(np.float64), [1.0]])
    ends = 2.0 / (n * (n - 1))
    weights = np.concatenate([[ends], w.astype(np.float64), [ends]])
    return nodes, weights


@dataclass
class Basis:
    n: int
    nodes: np.ndarray
    weights: np.ndarray
    vinv: np.ndarray  # inverse Vandermonde [s, j]
    invm: np.ndarray
    up: np.ndarray
    xi: np.ndarray  # [n, 2]


def make_basis(n) -> Basis:
    """DG matrices of ``main/basis.py:126-188``.  Legendre polynomials are evaluated from
    their power-series coefficients (``scipy.special.legendre``), the numerical route of the
    reference, so the tables agree with it to a few ulp."""
    x, w = lgl_nodes_weights(n)
    eig = [(2.0 * s + 1) / 2.0 for s in range(n - 1)] + [(n - 1) / 2.0]
    polys = [sp.legendre(s) for s in range(n)]
    dpolys = [p.deriv() for p in polys]
    vinv = np.array([[w[j] * eig[s] * polys[s](x[j]) for j in range(n)] for s in range(n)])
    pn1 = polys[n - 1](x)
    invm = np.diag(1.0 / w) + (n / 2) * np.outer(pn1, pn1)
    up = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            acc = 0
            for s in range(n):
                acc = acc + (2 * s + 1) / 2 * polys[s](x[i]) * dpolys[s](x[j])
            up[i, j] = w[j] * acc
    up[np.abs(up) < 1.0e-10] = 0.0
    xi = invm[:, [0, n - 1]].copy()
    return Basis(n=n, nodes=x, weights=w, vinv=vinv, invm=invm, up=up, xi=xi)


# ----------------------------------------------------------------------------------------------
# grids (main/grid.py:10-109)
# ----------------------------------------------------------------------------------------------
@dataclass
class Axis:
    low: float
    high: float
    res: int
    basis: Basis
    dx: float = 0.0
    J: float = 0.0
    arr: np.ndarray = None  # ghost-inclusive node coordinates (res+2, n)
    arr_max: float = 0.0
    # spectral (x only)
    wave_numbers: np.ndarray = None
    T: np.ndarray = None  # forward transform (res, n, M) complex
    P: np.ndarray = None  # inverse phases (M, res, n) complex


def make_axis(low, high, res, basis, spectrum=False) -> Axis:
    ax = Axis(low=low, high=high, res=int(res), basis=basis)
    length = high - low
    ax.dx = length / ax.res
    ax.J = 2.0 / ax.dx
    xl = np.linspace(low - ax.dx, high, num=ax.res + 2)
    xi01 = (np.array(basis.nodes) + 1) / 2
    ax.arr = xl[:, None] + ax.dx * xi01[None, :]
    ax.arr_max = np.amax(abs(ax.arr))
    if spectrum:
        nyq = 2.5 * length // ax.dx
        k1 = 2.0 * np.pi / length
        ax.wave_numbers = k1 * np.arange(1 - nyq, nyq)
        ax.P = np.exp(1j * np.multiply.outer(ax.wave_numbers, ax.arr[1:-1, :]))
        mid = np.array([(ax.arr[i, -1] + ax.arr[i, 0]) / 2.0 for i in range(1, ax.res + 1)])
        sgn = np.sign(ax.wave_numbers)
        sgn[ax.wave_numbers == 0] = 1.0
        n = basis.n
        ptilde = np.array([(sgn ** s) * np.exp(-1j * np.pi / 2.0 * s) *
                           sp.spherical_jn(s, np.absolute(ax.wave_numbers) / ax.J)
                           for s in range(n)])  # [s, m]
        ell = basis.vinv.T @ ptilde  # [j, m]
        phase = np.exp(-1j * np.multiply.outer(mid, ax.wave_numbers))  # [e, m]
        ax.T = phase[:, None, :] * ell[None, :, :]
    return ax


# Cockburn-Shu Courant numbers for RK3 (main/timestep.py:27), indexed by n - 1
COURANT_RK3 = [1.256, 0.409, 0.209, 0.130, 0.089, 0.066, 0.051, 0.040, 0.033]
RK3_COEFFS = np.array([[3 / 4, 1 / 4, 1 / 4], [1 / 3, 2 / 3, 2 / 3]])


@dataclass
class Case:
    """Everything the hot path needs for one problem instance."""

    n: int
    basis: Basis
    x: Axis
    u: Axis
    v: Axis
    accel: float
    B: float
    kappa: float
    qw: np.ndarray = None  # velocity quadrature weights (Nu, n, Nv, n) / (Ju Jv)
    xw: np.ndarray = None  # x quadrature weights (Nx, n)
    extra: dict = field(default_factory=dict)

    @property
    def shape(self):
        n = self.n
        return (self.x.res + 2, n, self.u.res + 2, n, self.v.res + 2, n)


def make_case(Nx, Nu, Nv, n, norm: Normalisation = None, om_pc=10.0, k=0.886, vmax=8.5,
              L=None) -> Case:
    """Reference driver geometry (``main/main.py:50-59``, ``main/main.py:122``)."""
    norm = norm or default_normalisation()
    b = make_basis(n)
    if L is None:
        k_est = k / om_pc
        L = 2.0 * np.pi / k_est
    lows = np.array([-L / 2.0, -vmax * norm.vt_e, -vmax * norm.vt_e])
    highs = np.array([L / 2.0, vmax * norm.vt_e, vmax * norm.vt_e])
    x = make_axis(lows[0], highs[0], Nx, b, spectrum=True)
    u = make_axis(lows[1], highs[1], Nu, b)
    v = make_axis(lows[2], highs[2], Nv, b)
    B = (norm.omp_e_tau / norm.omc_e_tau) / om_pc
    c = Case(n=n, basis=b, x=x, u=u, v=v, accel=norm.accel, B=B, kappa=norm.kappa)
    qu = np.multiply.outer(np.ones(Nu), b.weights)
    qv = np.multiply.outer(np.ones(Nv), b.weights)
    c.qw = np.multiply.outer(qu, qv) / (u.J * v.J)
    c.xw = np.multiply.outer(np.ones(Nx), b.weights)
    c.extra["norm"] = norm
    return c


# ----------------------------------------------------------------------------------------------
# initial conditions (main/grid.py:244-268 loss cone; perturbations)
# ----------------------------------------------------------------------------------------------
def loss_cone(case: Case, vt, ring_j):
    """Loss-cone ring f0 on every node including ghosts (main/grid.py:253-268)."""
    factor = 1.0 / ((2.0 ** ring_j) * (2.0 * np.pi) * (vt ** 2.0) * math.factorial(ring_j))
    rsq = (np.multiply.outer(case.u.arr ** 2.0, np.ones_like(case.v.arr)) +
           np.multiply.outer(np.ones_like(case.u.arr), case.v.arr ** 2.0)) / (vt ** 2.0)
    pol = (rsq ** ring_j) * np.exp(-0.5 * rsq)
    ones_x = np.ones((case.x.res + 2, case.n))
    return factor * np.multiply.outer(ones_x, pol)


def cos_perturbed(case: Case, vt, ring_j, amp, kx=None, noise=0.0, seed=0):
    """f0(u, v) * (1 + amp cos(k x) + noise * r(x)), r uniform in [-1, 1] per x node (seeded)."""
    f0 = loss_cone(case, vt, ring_j)
    kx = (2.0 * np.pi / (case.x.high - case.x.low)) if kx is None else kx
    mod = 1.0 + amp * np.cos(kx * case.x.arr)
    if noise:
        rng = np.random.default_rng(seed)
        r = rng.uniform(-1.0, 1.0, size=(case.x.res, case.n))
        rr = np.zeros_like(mod)
        rr[1:-1] = r
        rr[0] = r[-1]
        rr[-1] = r[0]
        mod = mod + noise * rr
    return f0 * mod[:, :, None, None, None, None]


# ----------------------------------------------------------------------------------------------
# RHS (main/fluxes.py:59-207)
# ----------------------------------------------------------------------------------------------
def _contract(mat, arr, axis):
    """out[.., i, ..] = sum_p mat[i, p] arr[.., p, ..] along ``axis``."""
    return np.moveaxis(np.tensordot(mat, arr, axes=([1], [axis])), 0, axis)


def _direction(F, pos, neg, up, xi, elem_axis, node_axis):
    n = up.shape[0]
    internal = _contract(up, F, node_axis)
    right = np.take(F, n - 1, axis=node_axis)  # face slabs, node axis removed
    left = np.take(F, 0, axis=node_axis)
    eaxis = elem_axis if elem_axis < node_axis else elem_axis - 1
    g_left = -(np.roll(right, 1, axis=eaxis) * pos + left * neg)
    g_right = right * pos + np.roll(left, -1, axis=eaxis) * neg
    lift = (np.expand_dims(g_left, node_axis) * _bcast(xi[:, 0], node_axis, F.ndim) +
            np.expand_dims(g_right, node_axis) * _bcast(xi[:, 1], node_axis, F.ndim))
    return internal - lift


def _bcast(vec, axis, ndim):
    shape = [1] * ndim
    shape[axis] = vec.shape[0]
    return vec.reshape(shape)


def rhs(f, E, case: Case):
    """Semi-discrete RHS on the ghost-inclusive array; ghost rows of the result are garbage
    (the caller slices the interior, as ``main/timestep.py:158-177`` does)."""
    b = case.basis
    a = case.accel
    ux = case.u.arr  # (U, n)
    vx = case.v.arr
    # x: speed u[a, j]
    sx = ux[None, None, :, :, None, None]
    Fx = f * sx
    px = (sx >= 0).astype(np.float64)
    nx = (sx < 0).astype(np.float64)
    out_x = _direction(Fx, px[:, 0], nx[:, 0], b.up, b.xi, 0, 1)
    # u: speed a (E[e, i] + B v[b, k])
    su = a * (E[:, :, None, None] + case.B * vx[None, None, :, :])  # (X, n, V, n)
    su6 = su[:, :, None, None, :, :]
    Fu = f * su6
    pu = (su6 >= 0).astype(np.float64)[:, :, :, 0]
    nu = (su6 < 0).astype(np.float64)[:, :, :, 0]
    out_u = _direction(Fu, pu, nu, b.up, b.xi, 2, 3)
    # v: speed a (-B u[a, j])
    sv = a * (-case.B * ux)
    sv6 = sv[None, None, :, :, None, None]
    Fv = f * sv6
    pv = (sv6 >= 0).astype(np.float64)[..., 0]
    nv = (sv6 < 0).astype(np.float64)[..., 0]
    out_v = _direction(Fv, pv, nv, b.up, b.xi, 4, 5)
    return out_x * case.x.J + out_u * case.u.J + out_v * case.v.J


# ----------------------------------------------------------------------------------------------
# moment, Poisson, energy, dt
# ----------------------------------------------------------------------------------------------
def moment_zero(f, case: Case):
    """rho[e, i] over interior elements (main/grid.py:319-321)."""
    inner = f[1:-1, :, 1:-1, :, 1:-1, :]
    return np.tensordot(inner, case.qw, axes=([2, 3, 4, 5], [0, 1, 2, 3]))


def poisson2(charge_density, case: Case):
    """Spectral Poisson solve (main/elliptic.py:117-145).  Returns (E ghost-inclusive
    (X, n), potential (Nx, n)).  The k = 0 mode is zeroed, which is what CuPy's complex
    division by zero followed by ``nan_to_num`` produces in the reference."""
    x = case.x
    rhs_ = case.kappa * charge_density
    c = np.tensordot(rhs_, x.T, axes=([0, 1], [0, 1])) * x.dx / (x.high - x.low)
    k = x.wave_numbers
    zero = k == 0
    ks = np.where(zero, 1.0, k)
    # -(c / (1j k)) = -(c_i / k) + 1j (c_r / k);  -(c / k^2)
    Ehat = (-(c.imag / ks)) + 1j * (c.real / ks)
    phihat = -(c / (ks ** 2.0))
    Ehat[zero] = 0.0
    phihat[zero] = 0.0
    E = np.zeros((x.res + 2, case.n))
    E[1:-1] = np.real(np.tensordot(Ehat, x.P, axes=([0], [0])))
    phi = np.real(np.tensordot(phihat, x.P, axes=([0], [0])))
    E[0] = E[-2]
    E[-1] = E[1]
    return E, phi


def electric_energy(E, case: Case):
    """0.5 sum w E^2 over interior nodes (main/elliptic.py:150-151)."""
    return 0.5 * np.tensordot(E[1:-1] ** 2.0, case.xw, axes=([0, 1], [0, 1]))


def max_speeds(E, case: Case):
    a, B = case.accel, case.B
    return np.absolute(np.array([case.u.arr_max,
                                 np.amax(np.absolute(a * E)) + abs(a * B * case.v.arr_max),
                                 a * abs(B * case.u.arr_max)]))


def adapt_dt(E, case: Case, courant=None):
    courant = COURANT_RK3[case.n - 1] if courant is None else courant
    ms = max_speeds(E, case)
    return courant / ((ms[0] / case.x.dx) + (ms[1] / case.u.dx) + (ms[2] / case.v.dx))


# ----------------------------------------------------------------------------------------------
# SSP-RK3 (main/timestep.py:141-187) and the main loop (main/timestep.py:81-103)
# ----------------------------------------------------------------------------------------------
INTERIOR = (slice(1, -1), slice(None), slice(1, -1), slice(None), slice(1, -1), slice(None))


def ssp_rk3_step(f, dt, case: Case):
    """One nonlinear SSP-RK3 step, in place on ``f`` (ghost-inclusive).

    Returns (E of the last Poisson solve, i.e. of stage s1; the new dt)."""
    f[0] = f[-2]
    f[-1] = f[1]
    stages = np.zeros((3,) + f.shape)
    stages[:, :, :, 0] = f[:, :, 0]
    stages[:, :, :, -1] = f[:, :, -1]
    stages[..., 0, :] = f[..., 0, :]
    stages[..., -1, :] = f[..., -1, :]
    rho = moment_zero(f, case)
    E, _ = poisson2(np.mean(rho) - rho, case)
    stages[0][INTERIOR] = f[INTERIOR] + dt * rhs(f, E, case)[INTERIOR]
    for i in (1, 2):
        s = stages[i - 1]
        s[0] = s[-2]
        s[-1] = s[1]
        rho = moment_zero(s, case)
        E, _ = poisson2(np.mean(rho) - rho, case)
        df = rhs(s, E, case)[INTERIOR]
        c = RK3_COEFFS[i - 1]
        stages[i][INTERIOR] = c[0] * f[INTERIOR] + c[1] * s[INTERIOR] + c[2] * dt * df
    dt_new = adapt_dt(E, case)
    f[INTERIOR] = stages[2][INTERIOR]
    return E, dt_new


@dataclass
class RunRecord:
    time_array: list
    field_energy: list
    dt_history: list
    steps: int


def run(f, case: Case, final_time=None, steps=None, E0=None):
    """The reference main loop: initial energy and dt from ``E0`` (the field the driver solved
    before the loop, ``main/main.py:131``), then steps while time < final_time (or a fixed
    number of steps).  ``f`` is advanced in place."""
    if E0 is None:
        rho = moment_zero(f, case)
        E0, _ = poisson2(rho - np.mean(rho), case)
    energy = [float(electric_energy(E0, case))]
    dt = adapt_dt(E0, case)
    t = 0.0
    times = [t]
    dts = [dt]
    count = 0
    while (steps is None and t < final_time) or (steps is not None and count < steps):
        E, dt = ssp_rk3_step(f, dt, case)
        t += dt
        count += 1
        times.append(t)
        dts.append(dt)
        energy.append(float(electric_energy(E, case)))
    return RunRecord(time_array=times, field_energy=energy, dt_history=dts, steps=count)


# ---------------------------------------------------------------------------------------------
# post-processing operators (main/grid.py:116-134, main/basis.py:291-317)
# ---------------------------------------------------------------------------------------------
def smooth_edges(arr):
    """In place: each interior element's face-node planes averaged with the neighbour's
    opposite face, x then u then v, left face then right face (``main/grid.py:116-134``); each
    statement sees the previous ones, the right-hand side of each is evaluated first."""
    r = np.roll
    a = arr
    a[1:-1, 0, 1:-1, :, 1:-1, :] = 0.5 * (r(a, 1, 0)[1:-1, -1, 1:-1, :, 1:-1, :] + a[1:-1, 0, 1:-1, :, 1:-1, :])
    a[1:-1, -1, 1:-1, :, 1:-1, :] = 0.5 * (r(a, -1, 0)[1:-1, 0, 1:-1, :, 1:-1, :] + a[1:-1, -1, 1:-1, :, 1:-1, :])
    a[1:-1, :, 1:-1, 0, 1:-1, :] = 0.5 * (r(a, 1, 2)[1:-1, :, 1:-1, -1, 1:-1, :] + a[1:-1, :, 1:-1, 0, 1:-1, :])
    a[1:-1, :, 1:-1, -1, 1:-1, :] = 0.5 * (r(a, -1, 2)[1:-1, :, 1:-1, 0, 1:-1, :] + a[1:-1, :, 1:-1, -1, 1:-1, :])
    a[1:-1, :, 1:-1, :, 1:-1, 0] = 0.5 * (r(a, 1, 4)[1:-1, :, 1:-1, :, 1:-1, -1] + a[1:-1, :, 1:-1, :, 1:-1, 0])
    a[1:-1, :, 1:-1, :, 1:-1, -1] = 0.5 * (r(a, -1, 4)[1:-1, :, 1:-1, :, 1:-1, 0] + a[1:-1, :, 1:-1, :, 1:-1, -1])
    return a


def fine_points(axis: "Axis", num=25):
    """25 equispaced points per element between its first and last node (``main/grid.py:38-42``)."""
    return np.array([np.linspace(axis.arr[i, 0], axis.arr[i, -1], num=num)
                     for i in range(1, axis.res + 1)])


def fine_lagrange(basis: "Basis", axis: "Axis", lim, num=25):
    """ell[e][i][p] = sum_s Vinv[s, i] P_s(xi_ep) for the elements lim[0] <= e < lim[1]
    (ghost-inclusive indices) at their fine points (``main/basis.py:296-309``)."""
    import scipy.special as sp

    fine = fine_points(axis, num)                       # interior elements 1..res
    mid = 0.5 * (axis.arr[1:-1, -1] + axis.arr[1:-1, 0])
    xi = axis.J * (fine[lim[0] - 1:lim[1] - 1, :] - mid[lim[0] - 1:lim[1] - 1, None])
    ps = np.array([sp.legendre(s)(xi) for s in range(basis.n)])
    return np.transpose(np.tensordot(basis.vinv, ps, axes=([0], [0])), [1, 0, 2])


def interpolate_values(arr, ell_x, ell_u, ell_v, limits):
    """Tensor-product interpolation of the nodal state on the fine points of an element range
    (``main/basis.py:310-317``): x, then u, then v contraction; out [ex, fx, eu, fu, ev, fv]."""
    x_lim, u_lim, v_lim = limits
    a = arr[x_lim[0]:x_lim[1], :, u_lim[0]:u_lim[1], :, v_lim[0]:v_lim[1], :]
    val = np.multiply(ell_x[:, :, :, None, None, None, None], a[:, :, None, :, :, :, :]).sum(axis=1)
    val = np.multiply(ell_u[None, None, :, :, :, None, None], val[:, :, :, :, None, :, :]).sum(axis=3)
    val = np.multiply(ell_v[None, None, None, None, :, :, :], val[:, :, :, :, :, :, None]).sum(axis=5)
    return val
