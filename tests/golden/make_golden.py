"""Generate golden fixtures by running the reference (crewsdw/Vlasov1D2V) on the CPU.

Run in a container that has the reference checkout, with ``VLASOV_REFERENCE_MAIN`` naming its
``main/`` directory (required; there is no default)::

    VLASOV_REFERENCE_MAIN=<checkout>/main python tests/golden/make_golden.py            # all
    VLASOV_REFERENCE_MAIN=<checkout>/main python tests/golden/make_golden.py basis tiny # a subset

The reference modules are imported unmodified through ``ref_shim`` (CuPy -> NumPy).  Every
array written here is produced by reference code; the only inputs built outside the reference
are the cos-perturbed loss-cone initial states of the ``cfg1`` case, which use the oracle's
``cos_perturbed`` (the hot path is IC-agnostic; the fixture stores a checksum of that state so
the tests can confirm they rebuilt the same input).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import ref_shim  # noqa: E402

R = ref_shim.install()
cp = sys.modules["cupy"]

from oracle import vlasov_oracle as vo  # noqa: E402

INNER = (slice(1, -1), slice(None), slice(1, -1), slice(None), slice(1, -1), slice(None))
MP = 1.67262158e-27
C = 299792458.0
E_CHARGE = 1.602176634e-19


def _refs():
    triplet = np.array([1.0e21, (MP * C ** 2.0) / E_CHARGE, 1.0])
    return R.reference.Reference(triplet=triplet, mass_fraction=1836.15267343)


def _np(x):
    return np.array(np.asarray(x))


def gen_basis():
    out = {}
    for n in range(1, 11):
        b = R.basis.Basis1D(n)
        out[f"n{n}_nodes"] = np.array(b.nodes, dtype=np.float64)
        out[f"n{n}_weights"] = np.array(b.weights, dtype=np.float64)
        out[f"n{n}_vinv"] = _np(b.vandermonde_inverse)
        out[f"n{n}_invm"] = _np(b.invm)
        out[f"n{n}_up"] = _np(b.up)
        out[f"n{n}_xi"] = _np(b.xi)
    out["courant_rk3"] = np.array(R.timestep.courant_numbers[3])
    np.savez_compressed(os.path.join(HERE, "basis.npz"), **out)


def _setup(res, order, om_pc=10.0, perturbation=True, delta_n=1.0e-3, ring_j=6):
    refs = _refs()
    orders = np.array([order] * 3)
    basis = R.basis.Basis3D(orders)
    k_est = 0.886 / om_pc
    L = 2.0 * np.pi / k_est
    lows = np.array([-L / 2.0, -8.5 * refs.vt_e, -8.5 * refs.vt_e])
    highs = np.array([L / 2.0, 8.5 * refs.vt_e, 8.5 * refs.vt_e])
    resolutions = np.array(res)
    grids = R.grid.Grid3D(basis=basis, lows=lows, highs=highs, resolutions=resolutions)
    f0 = R.grid.Distribution(vt=refs.vt_e, ring_j=ring_j, resolutions=resolutions, orders=orders,
                             om=-0.349j, om_pc=om_pc, delta_n=delta_n, perturbation=perturbation)
    f0.initialize_quad_weights(grids)
    f0.initialize_gpu(grids)
    el = R.elliptic.Elliptic(poisson_coefficient=refs.charge_density_multiplier)
    el.set_magnetic_field(magnetic_field=(refs.omp_e_tau / refs.omc_e_tau) / om_pc)
    flux = R.fluxes.DGFlux(resolutions=resolutions + 2, orders=orders,
                           flux_coefficients=refs.electron_acceleration_multiplier)
    st = R.timestep.Stepper(time_order=3, space_order=order, write_time=1.0e9, final_time=1.0e9)
    return dict(refs=refs, basis=basis, grids=grids, f=f0, el=el, flux=flux, st=st, L=L,
                lows=lows, highs=highs)


def _steps(s, nsteps, out, keep_every=1, keep_f=True):
    """The body of ``Stepper.main_loop`` (main/timestep.py:81-103) for a fixed step count."""
    st, el, grids, f = s["st"], s["el"], s["grids"], s["f"]
    energies = [float(el.electric_energy(grid=grids.x).get())]
    st.adapt_time_step(max_speeds=R.timestep.get_max_speeds(grids, el, s["refs"]),
                       dx=grids.x.dx, du=grids.u.dx, dv=grids.v.dx)
    dts = [st.dt]
    times = [0.0]
    t = 0.0
    for it in range(nsteps):
        st.nonlinear_ssp_rk(distribution=f, basis=s["basis"], elliptic=el, grids=grids,
                            dg_flux=s["flux"], refs=s["refs"])
        t += st.dt
        times.append(t)
        dts.append(st.dt)
        energies.append(float(el.electric_energy(grid=grids.x).get()))
        if keep_f and ((it + 1) % keep_every == 0 or it + 1 == nsteps):
            out[f"f_step{it + 1}"] = _np(f.arr)[INNER]
            out[f"E_step{it + 1}"] = _np(el.electric_field)
    out["energy"] = np.array(energies)
    out["dt"] = np.array(dts)
    out["time"] = np.array(times)


def gen_small(name, res, order, nsteps, seed):
    s = _setup(res, order)
    grids, el, f = s["grids"], s["el"], s["f"]
    out = {"res": np.array(res), "order": np.array(order), "L": np.array(s["L"]),
           "lows": s["lows"], "highs": s["highs"]}
    out["x_arr"] = _np(grids.x.arr)
    out["u_arr"] = _np(grids.u.arr)
    out["v_arr"] = _np(grids.v.arr)
    out["wave_numbers"] = _np(grids.x.wave_numbers)
    out["T"] = _np(grids.x.spectral_transform)
    out["P"] = _np(grids.x.grid_phases)
    out["accel"] = np.array(s["refs"].electron_acceleration_multiplier)
    out["kappa"] = np.array(s["refs"].charge_density_multiplier)
    out["B"] = np.array(el.magnetic_field)
    out["vt"] = np.array(s["refs"].vt_e)
    out["f_init"] = _np(f.arr)
    n0 = f.moment_zero()
    out["rho_init"] = _np(n0)
    el.poisson2(charge_density=cp.asarray(n0) - cp.mean(n0), grid=grids.x, basis=s["basis"].b1)
    out["E_init"] = _np(el.electric_field)
    out["phi_init"] = _np(el.potential)
    # RHS of the initial state with the initial field
    out["rhs_init"] = _np(s["flux"].semi_discrete_rhs(function=f.arr, elliptic=el,
                                                       basis=s["basis"], grids=grids))[INNER]
    # RHS of a random state with a random field (exercises every upwind branch)
    rng = np.random.default_rng(seed)
    f_rand = rng.standard_normal(f.arr.shape)
    E_rand = rng.standard_normal(el.electric_field.shape) * 4.0
    saved_E = el.electric_field
    el.electric_field = cp.asarray(E_rand)
    out["f_rand"] = f_rand
    out["E_rand"] = E_rand
    out["rhs_rand"] = _np(s["flux"].semi_discrete_rhs(function=cp.asarray(f_rand), elliptic=el,
                                                       basis=s["basis"], grids=grids))[INNER]
    # moment + poisson of the random state (charge density as the stepper forms it)
    rho_r = R.grid.Distribution.moment_zero_of_arr(f, cp.asarray(f_rand))
    out["rho_rand"] = _np(rho_r)
    el.poisson2(charge_density=cp.mean(rho_r) - rho_r, grid=grids.x, basis=s["basis"].b1)
    out["E_rand_solved"] = _np(el.electric_field)
    out["phi_rand_solved"] = _np(el.potential)
    out["energy_rand_solved"] = np.array(float(el.electric_energy(grid=grids.x).get()))
    el.electric_field = saved_E
    el.poisson2(charge_density=cp.asarray(n0) - cp.mean(n0), grid=grids.x, basis=s["basis"].b1)
    _steps(s, nsteps, out)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


def gen_steps(name, res, order, nsteps, delta_n):
    """SSP-RK3 steps of the reference from its eigenmode initial state with a large amplitude
    ``delta_n``: the density perturbation is then a sizeable fraction of the density, so the field
    (formed from rho - mean(rho)) keeps the relative rounding of rho and the energy history can be
    held to the 1e-12 bar pointwise."""
    s = _setup(res, order, delta_n=delta_n)
    grids, el, f = s["grids"], s["el"], s["f"]
    out = {"res": np.array(res), "order": np.array(order), "delta_n": np.array(delta_n)}
    out["f_init"] = _np(f.arr)
    n0 = f.moment_zero()
    out["rho_init"] = _np(n0)
    el.poisson2(charge_density=cp.asarray(n0) - cp.mean(n0), grid=grids.x, basis=s["basis"].b1)
    out["E_init"] = _np(el.electric_field)
    _steps(s, nsteps, out)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


def gen_cfg1(nsteps=200, out_name="cfg1_200", summary=True):
    """Config 1 of the benchmark set: Nx = Nu = Nv = 16, n = 8, loss cone j = 6 times
    (1 + 0.01 cos kx), nsteps SSP-RK3 steps.  Stores the energy/dt/time histories and a
    compact summary of the final state."""
    res = (16, 16, 16)
    order = 8
    s = _setup(res, order, perturbation=False)
    case = vo.make_case(*res, order)
    f_init = vo.cos_perturbed(case, s["refs"].vt_e, 6, 0.01)
    s["f"].arr = cp.asarray(f_init)
    n0 = s["f"].moment_zero()
    s["el"].poisson2(charge_density=cp.asarray(n0) - cp.mean(n0), grid=s["grids"].x,
                     basis=s["basis"].b1)
    out = {"f_init_sum": np.array(f_init.sum()), "f_init_sumsq": np.array((f_init ** 2).sum()),
           "f_init_probe": f_init[5, 3, 7, 2, 9, 4:8].copy()}
    t0 = time.time()
    _steps(s, nsteps, out, keep_f=False)
    out["seconds"] = np.array(time.time() - t0)
    out["blas_threads"] = np.array(int(os.environ.get("OPENBLAS_NUM_THREADS", "0")))
    if not summary:
        np.savez_compressed(os.path.join(HERE, f"{out_name}.npz"), **out)
        return
    f = _np(s["f"].arr)
    out["final_rho"] = _np(s["f"].moment_zero())
    out["final_E"] = _np(s["el"].electric_field)
    inner = f[1:-1, :, 1:-1, :, 1:-1, :]
    out["final_sum_x"] = inner.sum(axis=(2, 3, 4, 5))
    out["final_sum_u"] = inner.sum(axis=(0, 1, 4, 5))
    out["final_sum_v"] = inner.sum(axis=(0, 1, 2, 3))
    out["final_norm2"] = np.array(np.sqrt((inner ** 2).sum()))
    out["final_slice_xu"] = inner[:, :, :, :, 7, 3].copy()
    out["final_slice_uv"] = inner[6, 2].copy()
    np.savez_compressed(os.path.join(HERE, "cfg1_200.npz"), **out)


def gen_linear(res=(4, 6, 5), order=4, nsteps=2):
    """The DG central-flux Poisson solve (main/elliptic.py:24-115) of the initial density, and
    steps of the linear SSP-RK3 stepper (main/timestep.py:189-229) that uses it."""
    s = _setup(res, order)
    grids, el, f = s["grids"], s["el"], s["f"]
    el.build_central_flux_operator(grid=grids.x, basis=s["basis"].b1)
    el.invert()
    n0 = f.moment_zero()
    el.poisson(charge_density=cp.mean(n0) - n0, grid=grids.x, basis=s["basis"].b1)
    out = {"res": np.array(res), "order": order, "f_init": _np(f.arr), "rho_init": _np(n0),
           "E_dg": _np(el.electric_field), "phi_dg": _np(el.potential),
           "central_flux_operator": _np(el.central_flux_operator),
           "gradient_operator": _np(el.gradient_operator)}
    st = R.timestep.Stepper(time_order=3, space_order=order, write_time=1.0e9, final_time=1.0e9,
                            linear=True)
    st.adapt_time_step(max_speeds=R.timestep.get_max_speeds(grids, el, s["refs"]),
                       dx=grids.x.dx, du=grids.u.dx, dv=grids.v.dx)
    out["dt0"] = st.dt
    for it in range(nsteps):
        st.ssp_rk_update(distribution=f, basis=s["basis"], grids=grids, elliptic=el,
                         dg_flux=s["flux"], refs=s["refs"])
        out[f"f_step{it + 1}"] = _np(f.arr)
        out[f"E_step{it + 1}"] = _np(el.electric_field)
        out[f"dt_step{it + 1}"] = st.dt
    np.savez_compressed(os.path.join(HERE, "linear.npz"), **out)


def gen_post(res=(3, 3, 4), order=4, seed=5):
    """Post-processing operators of the reference on a random state: smooth_edges
    (main/grid.py:116-134) and Basis3D.interpolate_values (main/basis.py:291-317) on the
    fine points of an element sub-range."""
    refs = _refs()
    orders = np.array([order] * 3)
    basis = R.basis.Basis3D(orders)
    L = 2.0 * np.pi / (0.886 / 10.0)
    lows = np.array([-L / 2.0, -8.5 * refs.vt_e, -8.5 * refs.vt_e])
    highs = np.array([L / 2.0, 8.5 * refs.vt_e, 8.5 * refs.vt_e])
    grids = R.grid.Grid3D(basis=basis, lows=lows, highs=highs, resolutions=np.array(res),
                          fine_all=True)
    rng = np.random.default_rng(seed)
    shape = (res[0] + 2, order, res[1] + 2, order, res[2] + 2, order)
    state = rng.standard_normal(shape)
    smoothed = _np(R.grid.smooth_edges(cp.asarray(state.copy())))
    limits = np.array([[2, 3], [2, 3], [1, 3]])
    interp = _np(basis.interpolate_values(grids, state, limits))
    np.savez_compressed(os.path.join(HERE, "post.npz"), res=np.array(res), order=order,
                        state=state, smoothed=smoothed, limits=limits, interp=interp)


def main(argv):
    which = argv or ["basis", "tiny", "small", "n8", "n9", "tiny_p", "small_p", "n8_p", "n9_p", "cfg1",
                     "post", "linear"]
    if "basis" in which:
        gen_basis()
    if "tiny" in which:
        gen_small("tiny", (3, 4, 5), 3, 3, seed=1)
    if "small" in which:
        gen_small("small", (4, 6, 5), 4, 4, seed=2)
    if "n8" in which:
        gen_small("n8", (2, 2, 3), 8, 1, seed=3)
    if "n9" in which:
        gen_small("n9", (2, 2, 2), 9, 1, seed=4)
    # large-amplitude variants of the four cases: energy bar 1e-12 pointwise
    if "tiny_p" in which:
        gen_steps("tiny_p", (3, 4, 5), 3, 3, 0.3)
    if "small_p" in which:
        gen_steps("small_p", (4, 6, 5), 4, 4, 0.3)
    if "n8_p" in which:
        gen_steps("n8_p", (2, 2, 3), 8, 2, 10.0)
    if "n9_p" in which:
        gen_steps("n9_p", (2, 2, 2), 9, 2, 0.3)
    if "cfg1" in which:
        gen_cfg1()
    if "post" in which:
        gen_post()
    if "linear" in which:
        gen_linear()
    if "cfg1_noise" in which:
        # the same run with a different BLAS thread count: the reference's own summation-order
        # noise floor for the energy history (run with OPENBLAS_NUM_THREADS=1)
        gen_cfg1(out_name="cfg1_200_blas1", summary=False)


if __name__ == "__main__":
    main(sys.argv[1:])
