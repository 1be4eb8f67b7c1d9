"""GPU parity of the kernels around the loop: initial-state construction on the device,
smooth_edges and the fine-grid interpolation, against the reference's fixtures, the host
construction (bit-identical to the reference's) and the CPU oracle."""
import numpy as np
import pytest
import torch

from helpers import SMALL_CASES, case_setup, golden, rel_err
from oracle import vlasov_oracle as vo

pytestmark = pytest.mark.gpu


def _grids(res, n, fine_all=False):
    from vlasov1d2v_b200 import problem
    from vlasov1d2v_b200.basis import Basis3D
    from vlasov1d2v_b200.grid import Grid3D

    refs = problem.default_reference()
    basis = Basis3D(np.array([n] * 3))
    L = 2.0 * np.pi / (0.886 / 10.0)
    grids = Grid3D(basis, np.array([-L / 2, -8.5 * refs.vt_e, -8.5 * refs.vt_e]),
                   np.array([L / 2, 8.5 * refs.vt_e, 8.5 * refs.vt_e]), np.array(res),
                   fine_all=fine_all)
    return refs, basis, grids


@pytest.mark.parametrize("name", SMALL_CASES)
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_device_initial_state(cuda, name, precision):
    """Eigenmode-perturbed loss cone built by vl_initial_state == the reference's f_init
    (bit for bit in FP64; in FP32 the state is the rounded deviation from the FP64 loss cone)."""
    from vlasov1d2v_b200.grid import Distribution

    G, res, n = case_setup(name)
    refs, basis, grids = _grids(res, n)
    d = Distribution(vt=refs.vt_e, ring_j=6, resolutions=res, orders=[n] * 3, om=-0.349j,
                     om_pc=10.0, delta_n=1.0e-3, perturbation=True, precision=precision)
    d.initialize_gpu(grids)
    if precision == "fp64":
        np.testing.assert_array_equal(d.arr.get(), G["f_init"])
    else:
        pert = G["f_init"] - d.background[None, None]
        assert rel_err(d.arr.get(), pert) < 1e-7
        assert rel_err(d.full_array().get(), G["f_init"]) < 1e-8


def test_device_cos_initial_state(cuda):
    """Benchmark initial state f0 (1 + a cos kx + noise) on the device == the host product."""
    from vlasov1d2v_b200 import problem

    p = problem.build((4, 6, 5), 8, perturbation="cos", amp=1.0e-3, noise=1.0e-6, seed=3)
    host = problem.cos_perturbed(p.grids, p.refs.vt_e, 6, 1.0e-3, noise=1.0e-6, seed=3)
    np.testing.assert_array_equal(p.f.arr.get(), host)


def test_smooth_edges_matches_reference(cuda):
    from vlasov1d2v_b200.grid import smooth_edges

    G = golden("post")
    t = torch.as_tensor(G["state"].copy(), device="cuda")
    out = smooth_edges(t)
    np.testing.assert_array_equal(out.get(), G["smoothed"])
    # the oracle restatement agrees with both
    np.testing.assert_array_equal(vo.smooth_edges(G["state"].copy()), G["smoothed"])


def test_smooth_edges_odd_shapes_against_oracle(cuda):
    from vlasov1d2v_b200.grid import smooth_edges

    rng = np.random.default_rng(11)
    for shape in ((4, 3, 5, 3, 3, 3), (3, 5, 4, 5, 6, 5)):
        a = rng.standard_normal(shape)
        out = smooth_edges(torch.as_tensor(a.copy(), device="cuda")).get()
        np.testing.assert_array_equal(out, vo.smooth_edges(a.copy()))


def test_interpolate_values_matches_reference(cuda):
    G = golden("post")
    res, n = [int(r) for r in G["res"]], int(G["order"])
    refs, basis, grids = _grids(res, n, fine_all=True)
    lim = [tuple(int(v) for v in row) for row in G["limits"]]
    out = basis.interpolate_values(grids, torch.as_tensor(G["state"], device="cuda"), lim).get()
    assert out.shape == G["interp"].shape
    assert rel_err(out, G["interp"]) <= 1e-14
    host = basis.interpolate_values_host(grids, G["state"], lim)
    assert rel_err(out, host) <= 1e-14


def test_checkpoint_resume_is_exact(cuda, tmp_path):
    """3 + 3 steps in one set of objects, or 3 + checkpoint + resume in fresh objects + 3:
    identical (both make the same two loop calls, so the density summation order matches)."""
    from vlasov1d2v_b200 import data_management as dm
    from vlasov1d2v_b200 import problem

    def fresh():
        return problem.build((4, 6, 5), 4, perturbation="eigenmode", amp=1.0e-2)

    a = fresh()
    for _ in range(2):
        a.stepper.run_steps(a.f, a.basis, a.elliptic, a.grids, a.flux, a.refs, 3)
    b = fresh()
    b.stepper.run_steps(b.f, b.basis, b.elliptic, b.grids, b.flux, b.refs, 3)
    folder = str(tmp_path) + "/"
    geo = np.array([[b.lows[d], b.highs[d], b.resolutions[d], b.orders[d]] for d in range(3)])
    rd = dm.RunData(folder, "ck", b.f.shape, geo, np.array([1.0, 0.1, b.stepper.courant, 3]), b.refs)
    rd.save_checkpoint(b.f, b.elliptic, b.stepper)
    c = fresh()
    c.stepper.resume_from(dm.ReadData(folder, "ck").read_checkpoint(), c.f, c.elliptic)
    c.stepper.run_steps(c.f, c.basis, c.elliptic, c.grids, c.flux, c.refs, 3)
    np.testing.assert_array_equal(c.f.arr.get(), a.f.arr.get())
    np.testing.assert_array_equal(c.stepper.field_energy, a.stepper.field_energy)
    np.testing.assert_array_equal(c.stepper.time_array, a.stepper.time_array)
    assert c.stepper.steps_counter == a.stepper.steps_counter == 6


def test_dg_poisson_and_linear_stepper_match_reference(cuda):
    """Elliptic.poisson (central-flux DG with anti-aliasing) of the initial density and two steps
    of the linear SSP-RK3 stepper, against the reference's fixture."""
    from helpers import F_RTOL, field_rtol
    from vlasov1d2v_b200 import problem
    from vlasov1d2v_b200.timestep import Stepper, get_max_speeds

    G = golden("linear")
    res, n = tuple(int(r) for r in G["res"]), int(G["order"])
    p = problem.build(res, n)
    np.testing.assert_array_equal(p.f.arr.get(), G["f_init"])
    el = p.elliptic
    el.build_central_flux_operator(grid=p.grids.x, basis=p.basis.b1)
    el.invert()
    rho = p.f.moment_zero()
    el.poisson(charge_density=rho.mean() - rho, grid=p.grids.x, basis=p.basis.b1)
    tol = field_rtol(G["rho_init"])
    assert rel_err(el.electric_field.get(), G["E_dg"]) < tol
    assert rel_err(el.potential.get(), G["phi_dg"]) < tol
    st = Stepper(time_order=3, space_order=n, write_time=1e9, final_time=1e9, linear=True)
    st.adapt_time_step(get_max_speeds(p.grids, el, p.refs), p.grids.x.dx, p.grids.u.dx, p.grids.v.dx)
    assert abs(st.dt - float(G["dt0"])) <= 1e-13 * float(G["dt0"])
    for it in (1, 2):
        st.ssp_rk_update(distribution=p.f, basis=p.basis, grids=p.grids, elliptic=el, dg_flux=p.flux,
                         refs=p.refs)
        inner = (slice(1, -1), slice(None), slice(1, -1), slice(None), slice(1, -1), slice(None))
        assert rel_err(p.f.arr.get()[inner], G[f"f_step{it}"][inner]) < F_RTOL
        assert rel_err(el.electric_field.get(), G[f"E_step{it}"]) < tol
        assert abs(st.dt - float(G[f"dt_step{it}"])) <= 1e-12 * st.dt
