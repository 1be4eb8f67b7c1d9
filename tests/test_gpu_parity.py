"""GPU parity of the CUDA path (through the C ABI) against the reference's fixtures and the
CPU oracle.  FP64 plain form: f within 1e-12 relative, energies within the density-cancellation
aware bar of ``helpers.field_rtol`` (1e-12 unless the density perturbation is so small that
rounding of the density itself is amplified past it)."""
import numpy as np
import pytest
import torch

from helpers import F_RTOL, INNER, SMALL_CASES, case_setup, field_rtol, golden, history_err, rel_err
from oracle import vlasov_oracle as vo

pytestmark = pytest.mark.gpu


def _build(name, **kw):
    from vlasov1d2v_b200 import problem

    G, res, n = case_setup(name)
    p = problem.build(res, n, **kw)
    return G, p


def _np(t):
    return t.get() if hasattr(t, "get") else t.detach().cpu().numpy()


@pytest.mark.parametrize("name", SMALL_CASES)
def test_initial_state_and_field(cuda, name):
    G, p = _build(name)
    np.testing.assert_array_equal(_np(p.f.arr), G["f_init"])
    rho = _np(p.f.moment_zero())
    assert rel_err(rho, G["rho_init"]) < 1e-14
    assert rel_err(_np(p.elliptic.electric_field), G["E_init"]) < field_rtol(G["rho_init"])


@pytest.mark.parametrize("name", SMALL_CASES)
def test_rhs_matches_reference(cuda, name):
    G, p = _build(name)
    E_ref = G["E_init"]
    # the reference evaluated this RHS with its own initial field: use exactly that field
    p.elliptic.electric_field = torch.as_tensor(E_ref, device="cuda")
    r = _np(p.flux.semi_discrete_rhs(function=p.f.arr, elliptic=p.elliptic, basis=p.basis,
                                     grids=p.grids))[INNER]
    assert rel_err(r, G["rhs_init"]) < 1e-12
    p.elliptic.electric_field = torch.as_tensor(G["E_rand"], device="cuda")
    r = _np(p.flux.semi_discrete_rhs(function=torch.as_tensor(G["f_rand"], device="cuda"),
                                     elliptic=p.elliptic, basis=p.basis, grids=p.grids))[INNER]
    assert rel_err(r, G["rhs_rand"]) < 1e-13


@pytest.mark.parametrize("name", SMALL_CASES)
def test_directional_fluxes_sum_to_rhs(cuda, name):
    G, p = _build(name)
    p.elliptic.electric_field = torch.as_tensor(G["E_rand"], device="cuda")
    f = torch.as_tensor(G["f_rand"], device="cuda")
    kw = dict(function=f, basis=p.basis)
    fx = _np(p.flux.x_flux(grid_u=p.grids.u, elliptic=p.elliptic, grids=p.grids, **kw))
    fu = _np(p.flux.u_flux(elliptic=p.elliptic, grid_v=p.grids.v, grids=p.grids, **kw))
    fv = _np(p.flux.v_flux(elliptic=p.elliptic, grid_u=p.grids.u, grids=p.grids, **kw))
    tot = fx * p.grids.x.J + fu * p.grids.u.J + fv * p.grids.v.J
    assert rel_err(tot[INNER], G["rhs_rand"]) < 1e-13


@pytest.mark.parametrize("name", SMALL_CASES)
def test_moment_poisson_energy(cuda, name):
    G, p = _build(name)
    f = torch.as_tensor(G["f_rand"], device="cuda")
    rho = _np(p.f.moment_zero_of_arr(f))
    assert rel_err(rho, G["rho_rand"]) < 1e-14
    rho_t = torch.as_tensor(G["rho_rand"], device="cuda")
    p.elliptic.poisson2(charge_density=torch.mean(rho_t) - rho_t, grid=p.grids.x, basis=p.basis.b1)
    tol = field_rtol(G["rho_rand"])
    assert rel_err(_np(p.elliptic.electric_field), G["E_rand_solved"]) < tol
    assert rel_err(_np(p.elliptic.potential), G["phi_rand_solved"]) < tol
    W = float(p.elliptic.electric_energy(grid=p.grids.x).get())
    assert abs(W / float(G["energy_rand_solved"]) - 1) < 2 * tol


@pytest.mark.parametrize("name", SMALL_CASES)
def test_steps_match_reference(cuda, name):
    G, p = _build(name)
    nst = len(G["energy"]) - 1
    p.stepper.run_steps(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, nst)
    tol = field_rtol(G["rho_init"])
    np.testing.assert_allclose(p.stepper.field_energy, G["energy"], rtol=2 * tol, atol=0)
    np.testing.assert_allclose(p.stepper.time_array, G["time"], rtol=1e-14, atol=0)
    assert abs(p.stepper.dt / G["dt"][-1] - 1) < 1e-14
    assert rel_err(_np(p.f.arr)[INNER], G[f"f_step{nst}"]) < F_RTOL
    assert rel_err(_np(p.elliptic.electric_field), G[f"E_step{nst}"]) < tol


@pytest.mark.parametrize("name", ("tiny", "small"))
def test_main_loop_and_single_step_api(cuda, name):
    G, p = _build(name)
    nst = len(G["energy"]) - 1
    # main_loop until final_time: run to just past the golden's last time
    p.stepper.final_time = float(G["time"][nst - 1]) + 1e-12
    p.stepper.batch_steps = 2  # exercise several batches and the graph replay path
    p.stepper.main_loop(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, None)
    assert p.stepper.steps_counter == nst
    tol = field_rtol(G["rho_init"])
    np.testing.assert_allclose(p.stepper.field_energy, G["energy"], rtol=2 * tol, atol=0)
    assert rel_err(_np(p.f.arr)[INNER], G[f"f_step{nst}"]) < F_RTOL
    # the single-step API reproduces the first step
    G2, q = _build(name)
    st = q.stepper
    st.field_energy = np.append(st.field_energy, q.elliptic.electric_energy(grid=q.grids.x).get())
    from vlasov1d2v_b200.timestep import get_max_speeds

    st.adapt_time_step(get_max_speeds(q.grids, q.elliptic, q.refs), q.grids.x.dx, q.grids.u.dx,
                       q.grids.v.dx)
    # dt comes from max|a E| of the initial field, itself within rounding of the reference's
    assert abs(st.dt / G2["dt"][0] - 1) < 1e-14
    st.nonlinear_ssp_rk(q.f, q.basis, q.elliptic, q.grids, q.flux, q.refs)
    assert abs(st.dt / G2["dt"][1] - 1) < 1e-14
    assert rel_err(_np(q.f.arr)[INNER], G2["f_step1"]) < F_RTOL


@pytest.mark.parametrize("name", ("tiny_p", "small_p", "n8_p", "n9_p"))
def test_steps_match_reference_energy_1e12(cuda, name):
    """The four cases again with a large eigenmode amplitude (the density perturbation is a
    sizeable fraction of the density, so no cancellation amplifies its rounding into the field):
    f, E and the field energy of every step within 1e-12 relative of the reference, pointwise."""
    from vlasov1d2v_b200 import problem

    G = golden(name)
    res = tuple(int(r) for r in G["res"])
    n = int(G["order"])
    assert field_rtol(G["rho_init"]) == F_RTOL
    p = problem.build(res, n, amp=float(G["delta_n"]))
    np.testing.assert_array_equal(_np(p.f.arr), G["f_init"])
    assert rel_err(_np(p.elliptic.electric_field), G["E_init"]) < F_RTOL
    nst = len(G["energy"]) - 1
    p.stepper.run_steps(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, nst)
    np.testing.assert_allclose(p.stepper.field_energy, G["energy"], rtol=F_RTOL, atol=0)
    # dt (hence the clock) follows max |a E|, which dominates the speeds at this amplitude and
    # carries the field's rounding (measured 2.8e-14 at n = 8)
    np.testing.assert_allclose(p.stepper.time_array, G["time"], rtol=1e-13, atol=0)
    assert rel_err(_np(p.f.arr)[INNER], G[f"f_step{nst}"]) < F_RTOL
    assert rel_err(_np(p.elliptic.electric_field), G[f"E_step{nst}"]) < F_RTOL


def test_main_loop_energy_1e12(cuda):
    """Stepper.main_loop (batches, graph replay) on the large-amplitude case: energy history
    within 1e-12 relative of the reference at every step."""
    from vlasov1d2v_b200 import problem

    G = golden("small_p")
    p = problem.build(tuple(int(r) for r in G["res"]), int(G["order"]), amp=float(G["delta_n"]))
    nst = len(G["energy"]) - 1
    p.stepper.final_time = float(G["time"][nst - 1]) + 1e-12
    p.stepper.batch_steps = 3
    p.stepper.main_loop(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, None)
    assert p.stepper.steps_counter == nst
    np.testing.assert_allclose(p.stepper.field_energy, G["energy"], rtol=F_RTOL, atol=0)
    assert rel_err(_np(p.f.arr)[INNER], G[f"f_step{nst}"]) < F_RTOL


def test_x_ghost_swap_matches_reference(cuda):
    """After a step the reference's f holds, in its x-ghost slabs, the periodic copy taken at the
    start of that step (main/timestep.py:143); the device loop refreshes them the same way."""
    G, p = _build("small")
    f0 = _np(p.f.arr).copy()
    p.stepper.run_steps(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, 1)
    f1 = _np(p.f.arr)
    np.testing.assert_array_equal(f1[0], f0[-2])
    np.testing.assert_array_equal(f1[-1], f0[1])


@pytest.mark.parametrize("n", [1, 2, 3, 5, 6, 7, 10])
@pytest.mark.parametrize("precision", ["fp64"])
def test_rhs_against_oracle_all_orders(cuda, n, precision):
    """Random states on odd-sized grids for orders the fixtures do not cover."""
    from vlasov1d2v_b200 import problem

    res = (3, 2, 5) if n < 7 else (2, 2, 3)
    p = problem.build(res, n, perturbation=None, amp=0.0)
    c = vo.make_case(*res, n)
    rng = np.random.default_rng(100 + n)
    f = rng.standard_normal(c.shape)
    E = rng.standard_normal((res[0] + 2, n))
    p.elliptic.electric_field = torch.as_tensor(E, device="cuda")
    r = _np(p.flux.semi_discrete_rhs(function=torch.as_tensor(f, device="cuda"),
                                     elliptic=p.elliptic, basis=p.basis, grids=p.grids))[INNER]
    assert rel_err(r, vo.rhs(f, E, c)[INNER]) < 1e-13
    rho = _np(p.f.moment_zero_of_arr(torch.as_tensor(f, device="cuda")))
    assert rel_err(rho, vo.moment_zero(f, c)) < 1e-13


@pytest.mark.parametrize("n", [3, 5, 7, 9])
def test_odd_orders_on_aligned_rows(cuda, n):
    """Odd orders on an even number of v elements: the rows hold (nv + 2) n doubles, an even
    count, so the FP64 stage kernel runs in its TMA form (odd rows are only 8-byte aligned on
    other grids).  RHS of a random state and the three RK stage kinds against the oracle."""
    from vlasov1d2v_b200 import _lib, problem
    from vlasov1d2v_b200.context import get_context

    res = (2, 3, 4)
    p = problem.build(res, n, perturbation=None, amp=0.0)
    c = vo.make_case(*res, n)
    rng = np.random.default_rng(300 + n)
    f = rng.standard_normal(c.shape)
    E = rng.standard_normal((res[0] + 2, n))
    p.elliptic.electric_field = torch.as_tensor(E, device="cuda")
    r = _np(p.flux.semi_discrete_rhs(function=torch.as_tensor(f, device="cuda"),
                                     elliptic=p.elliptic, basis=p.basis, grids=p.grids))[INNER]
    R = vo.rhs(f, E, c)
    assert rel_err(r, R[INNER]) < 1e-13
    ctx = get_context(p.grids, accel=p.refs.electron_acceleration_multiplier,
                      bfield=p.elliptic.magnetic_field, kappa=p.elliptic.poisson_coefficient,
                      courant=p.stepper.courant)
    fin = f.copy()
    fin[0], fin[-1] = fin[-2], fin[1]  # periodic x ghosts: stage semantics
    R = vo.rhs(fin, E, c)
    fn = rng.standard_normal(c.shape)
    dt = 0.0071
    tin = torch.as_tensor(fin, device="cuda")
    tfn = torch.as_tensor(fn, device="cuda")
    tE = torch.as_tensor(E, device="cuda")
    tdt = torch.tensor([dt], dtype=torch.float64, device="cuda")
    for stage, want in ((0, fin + dt * R), (1, 0.75 * fn + 0.25 * fin + (0.25 * dt) * R),
                        (2, fn / 3 + (2 / 3) * fin + ((2 / 3) * dt) * R)):
        out = torch.zeros_like(tin)
        ctx.rk_stage(stage, tin, tfn if stage else None, out, tE, tdt, xhalo=_lib.VL_XHALO_PERIODIC,
                     partials=ctx.workspace)
        assert rel_err(_np(out)[INNER], want[INNER]) < 1e-14


@pytest.mark.parametrize("form", ["pencil", "tma"])
@pytest.mark.parametrize("res", [(2, 2, 3), (2, 2, 4), (2, 2, 2), (2, 3, 6)])
@pytest.mark.parametrize("n", [3, 5, 6, 7, 9])
def test_fp32_stage_kernels_other_orders(cuda, n, res, form, monkeypatch):
    """FP32 orders other than 4 and 8: the generic kernel's TMA form (the default where the rows
    are 16-byte multiples, (nv + 2) n a multiple of 4; the register-pencil kernel elsewhere) and
    the register-pencil kernel everywhere (VLASOV1D2V_STAGE_KERNEL=pencil).  The three RK stage
    kinds of a random state against the FP64 oracle, within FP32 rounding of the stage results.
    The switch is read when the context is created."""
    from vlasov1d2v_b200 import _lib, problem
    from vlasov1d2v_b200.context import get_context

    for var in ("VLASOV1D2V_GEN_NO_TMA", "VLASOV1D2V_STAGE_KERNEL"):
        monkeypatch.delenv(var, raising=False)
    if form == "pencil":
        monkeypatch.setenv("VLASOV1D2V_STAGE_KERNEL", "pencil")
    p = problem.build(res, n, perturbation=None, amp=0.0, precision="fp32")
    c = vo.make_case(*res, n)
    ctx = get_context(p.grids, precision="fp32", accel=p.refs.electron_acceleration_multiplier,
                      bfield=p.elliptic.magnetic_field, kappa=p.elliptic.poisson_coefficient,
                      courant=p.stepper.courant)
    rng = np.random.default_rng(500 + n + res[2])
    fin = rng.standard_normal(c.shape).astype(np.float32).astype(np.float64)
    fin[0], fin[-1] = fin[-2], fin[1]  # periodic x ghosts: stage semantics
    fn = rng.standard_normal(c.shape).astype(np.float32).astype(np.float64)
    E = rng.standard_normal((res[0] + 2, n))
    R = vo.rhs(fin, E, c)
    dt = 0.0071
    tin = torch.as_tensor(fin, dtype=torch.float32, device="cuda")
    tfn = torch.as_tensor(fn, dtype=torch.float32, device="cuda")
    tE = torch.as_tensor(E, device="cuda")
    tdt = torch.tensor([dt], dtype=torch.float64, device="cuda")
    for stage, want in ((0, fin + dt * R), (1, 0.75 * fn + 0.25 * fin + (0.25 * dt) * R),
                        (2, fn / 3 + (2 / 3) * fin + ((2 / 3) * dt) * R)):
        out = torch.zeros_like(tin)
        ctx.rk_stage(stage, tin, tfn if stage else None, out, tE, tdt, xhalo=_lib.VL_XHALO_PERIODIC,
                     partials=ctx.workspace)
        assert rel_err(_np(out).astype(np.float64)[INNER], want[INNER]) < 1e-5


def test_rk_stage_entry_point(cuda):
    """vl_rk_stage (one fused stage) against the oracle's stage formula."""
    from vlasov1d2v_b200 import _lib, problem
    from vlasov1d2v_b200.context import get_context

    res, n = (3, 4, 5), 4
    p = problem.build(res, n, perturbation=None)
    c = vo.make_case(*res, n)
    rng = np.random.default_rng(7)
    fin = rng.standard_normal(c.shape)
    fn = rng.standard_normal(c.shape)
    E = rng.standard_normal((res[0] + 2, n))
    fin[0], fin[-1] = fin[-2], fin[1]  # periodic x ghosts: stage semantics
    ctx = get_context(p.grids, accel=p.refs.electron_acceleration_multiplier,
                      bfield=p.elliptic.magnetic_field, kappa=p.elliptic.poisson_coefficient,
                      courant=p.stepper.courant)
    dt = 0.0123
    tin = torch.as_tensor(fin, device="cuda")
    tfn = torch.as_tensor(fn, device="cuda")
    tE = torch.as_tensor(E, device="cuda")
    tdt = torch.tensor([dt], dtype=torch.float64, device="cuda")
    R = vo.rhs(fin, E, c)
    for stage, want in ((0, fin + dt * R), (1, 0.75 * fn + 0.25 * fin + (0.25 * dt) * R),
                        (2, fn / 3 + (2 / 3) * fin + ((2 / 3) * dt) * R)):
        out = torch.zeros_like(tin)
        ctx.rk_stage(stage, tin, tfn if stage else None, out, tE, tdt, xhalo=_lib.VL_XHALO_PERIODIC,
                     partials=ctx.workspace)
        assert rel_err(_np(out)[INNER], want[INNER]) < 1e-14


@pytest.mark.slow
def test_cfg1_200_steps(cuda):
    """Config 1 of the benchmark set (16^3 elements, n = 8, loss cone j = 6 times
    1 + 0.01 cos kx): 200 SSP-RK3 steps against the reference's energy/dt/time histories and
    final-state summaries."""
    from vlasov1d2v_b200 import problem

    G = golden("cfg1_200")
    p = problem.build((16, 16, 16), 8, perturbation="cos", amp=0.01, batch_steps=50)
    assert float(_np(p.f.arr).sum()) == float(G["f_init_sum"])
    p.stepper.run_steps(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, 200)
    en = np.asarray(p.stepper.field_energy)
    # normwise over the history (the energy dips to 3e-7 of its peak near step 157)
    err_e = history_err(en, G["energy"])
    assert err_e < 1e-12, err_e
    # the reference's own spread (8 vs 1 BLAS threads) is of the same order
    noise = history_err(golden("cfg1_200_blas1")["energy"], G["energy"])
    assert noise < 1e-12
    np.testing.assert_allclose(p.stepper.time_array, G["time"], rtol=1e-13)
    f = _np(p.f.arr)[INNER]
    assert rel_err(f[:, :, :, :, 7, 3], G["final_slice_xu"]) < F_RTOL
    assert rel_err(f[6, 2], G["final_slice_uv"]) < F_RTOL
    assert abs(np.sqrt((f ** 2).sum()) / G["final_norm2"] - 1) < F_RTOL
    assert rel_err(_np(p.f.moment_zero()), G["final_rho"]) < 1e-13
