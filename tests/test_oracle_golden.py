"""Pin the CPU oracle against fixtures generated by the reference itself (tests/golden).

The fixtures come from ``tests/golden/make_golden.py``, which runs crewsdw/Vlasov1D2V's own
modules on the CPU.  These tests need no GPU.
"""
import numpy as np
import pytest

from helpers import INNER, SMALL_CASES, case_setup, field_rtol, golden, rel_err
from oracle import vlasov_oracle as vo


def test_basis_tables():
    """The oracle computes LGL constants in extended precision (correctly rounded); the
    reference evaluates sqrt(1/5), sqrt(3/7), ... in double for n <= 6, so nodes may differ by
    an ulp there.  Matrices agree to 1e-13."""
    g = golden("basis")
    for n in range(1, 11):
        b = vo.make_basis(n)
        np.testing.assert_allclose(b.nodes, g[f"n{n}_nodes"], rtol=0, atol=2.3e-16)
        np.testing.assert_allclose(b.weights, g[f"n{n}_weights"], rtol=5e-16, atol=0)
        for key, mine in (("vinv", b.vinv), ("invm", b.invm), ("up", b.up), ("xi", b.xi)):
            ref = g[f"n{n}_{key}"]
            assert np.max(np.abs(mine - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref))), (n, key)
    np.testing.assert_array_equal(vo.COURANT_RK3, g["courant_rk3"])


@pytest.mark.parametrize("name", SMALL_CASES)
def test_grid_and_dft_tables(name):
    G, res, n = case_setup(name)
    c = vo.make_case(*res, n)
    np.testing.assert_array_equal(c.x.arr, G["x_arr"])
    np.testing.assert_array_equal(c.u.arr, G["u_arr"])
    np.testing.assert_array_equal(c.v.arr, G["v_arr"])
    np.testing.assert_array_equal(c.x.wave_numbers, G["wave_numbers"])
    np.testing.assert_array_equal(c.x.T, G["T"])
    np.testing.assert_array_equal(c.x.P, G["P"])
    assert c.accel == G["accel"] and c.kappa == G["kappa"] and c.B == G["B"]


@pytest.mark.parametrize("name", SMALL_CASES)
def test_rhs(name):
    G, res, n = case_setup(name)
    c = vo.make_case(*res, n)
    assert rel_err(vo.rhs(G["f_init"], G["E_init"], c)[INNER], G["rhs_init"]) < 1e-12
    assert rel_err(vo.rhs(G["f_rand"], G["E_rand"], c)[INNER], G["rhs_rand"]) < 1e-13


@pytest.mark.parametrize("name", SMALL_CASES)
def test_moment_poisson_energy(name):
    G, res, n = case_setup(name)
    c = vo.make_case(*res, n)
    rho = vo.moment_zero(G["f_rand"], c)
    assert rel_err(rho, G["rho_rand"]) < 1e-14
    E, phi = vo.poisson2(np.mean(rho) - rho, c)
    tol = field_rtol(G["rho_rand"])
    assert rel_err(E, G["E_rand_solved"]) < tol
    assert rel_err(phi, G["phi_rand_solved"]) < tol
    assert abs(vo.electric_energy(E, c) / G["energy_rand_solved"] - 1) < 2 * tol
    rho0 = vo.moment_zero(G["f_init"], c)
    assert rel_err(rho0, G["rho_init"]) < 1e-14
    E0, _ = vo.poisson2(rho0 - np.mean(rho0), c)
    assert rel_err(E0, G["E_init"]) < field_rtol(G["rho_init"])


@pytest.mark.parametrize("name", SMALL_CASES)
def test_steps(name):
    G, res, n = case_setup(name)
    c = vo.make_case(*res, n)
    f = G["f_init"].copy()
    nst = len(G["energy"]) - 1
    rho0 = vo.moment_zero(f, c)
    E0, _ = vo.poisson2(rho0 - np.mean(rho0), c)
    rec = vo.run(f, c, steps=nst, E0=E0)
    tol = field_rtol(G["rho_init"])
    np.testing.assert_allclose(rec.field_energy, G["energy"], rtol=2 * tol, atol=0)
    np.testing.assert_allclose(rec.dt_history, G["dt"], rtol=1e-14, atol=0)
    np.testing.assert_allclose(rec.time_array, G["time"], rtol=1e-14, atol=0)
    assert rel_err(f[INNER], G[f"f_step{nst}"]) < 1e-12


@pytest.mark.parametrize("name", ("tiny_p", "small_p", "n8_p", "n9_p"))
def test_steps_large_amplitude(name):
    """The large-amplitude fixtures: energy of every step within 1e-12 relative, pointwise."""
    G = golden(name)
    res = tuple(int(r) for r in G["res"])
    n = int(G["order"])
    c = vo.make_case(*res, n)
    f = G["f_init"].copy()
    nst = len(G["energy"]) - 1
    rec = vo.run(f, c, steps=nst, E0=G["E_init"])
    np.testing.assert_allclose(rec.field_energy, G["energy"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(rec.time_array, G["time"], rtol=1e-14, atol=0)
    assert rel_err(f[INNER], G[f"f_step{nst}"]) < 1e-12


def test_cfg1_first_steps():
    """Config 1 (16^3 elements, n = 8, 1 + 0.01 cos kx): three oracle steps against the first
    entries of the reference's 200-step histories."""
    G = golden("cfg1_200")
    c = vo.make_case(16, 16, 16, 8)
    f = vo.cos_perturbed(c, c.extra["norm"].vt_e, 6, 0.01)
    assert f.sum() == G["f_init_sum"]
    np.testing.assert_array_equal(f[5, 3, 7, 2, 9, 4:8], G["f_init_probe"])
    rec = vo.run(f, c, steps=3)
    np.testing.assert_allclose(rec.field_energy, G["energy"][:4], rtol=1e-12)
    np.testing.assert_allclose(rec.dt_history, G["dt"][:4], rtol=1e-14)
    np.testing.assert_allclose(rec.time_array, G["time"][:4], rtol=1e-14)


def test_cfg1_reference_noise_floor():
    """The reference run twice with different BLAS thread counts: its energy histories agree
    normwise to well below the 1e-12 parity bar (the floor any reimplementation sits on)."""
    from helpers import history_err

    a, b = golden("cfg1_200"), golden("cfg1_200_blas1")
    assert history_err(b["energy"], a["energy"]) < 1e-13
    np.testing.assert_allclose(b["time"], a["time"], rtol=1e-14)


def test_post_processing_operators():
    """smooth_edges and Basis3D.interpolate_values of the reference, pinned on a random state."""
    G = golden("post")
    res, n = [int(r) for r in G["res"]], int(G["order"])
    assert np.array_equal(vo.smooth_edges(G["state"].copy()), G["smoothed"])
    c = vo.make_case(*res, n)
    lim = G["limits"]
    ells = [vo.fine_lagrange(c.basis, ax, lim[d]) for d, ax in enumerate((c.x, c.u, c.v))]
    out = vo.interpolate_values(G["state"], *ells, lim)
    assert rel_err(out, G["interp"]) <= 1e-14


def test_central_flux_operator_matches_reference():
    """The DG central-flux Laplacian and gradient map (main/elliptic.py:24-81), assembled here as
    block linear maps, against the reference's own matrices (probed node by node there)."""
    from vlasov1d2v_b200.basis import Basis3D
    from vlasov1d2v_b200.elliptic import central_flux_matrices
    from vlasov1d2v_b200.grid import Grid1D

    G = golden("linear")
    res, n = tuple(int(r) for r in G["res"]), int(G["order"])
    L = 2.0 * np.pi / (0.886 / 10.0)
    basis = Basis3D(np.array([n] * 3))
    grid = Grid1D(-L / 2.0, L / 2.0, res[0], basis.b1, spectrum=True)
    op, grad = central_flux_matrices(grid, basis.b1)
    ref_op, ref_grad = G["central_flux_operator"], G["gradient_operator"]
    assert op.shape == ref_op.shape and grad.shape == ref_grad.shape
    scale = np.max(np.abs(ref_op))
    assert np.max(np.abs(op - ref_op)) <= 1e-14 * scale
    assert np.max(np.abs(grad - ref_grad)) <= 1e-14 * np.max(np.abs(ref_grad))
    # the inverse the solve applies agrees to the conditioning of the bordered system
    inv, ref_inv = np.linalg.inv(op), np.linalg.inv(ref_op)
    assert np.max(np.abs(inv - ref_inv)) <= 1e-10 * np.max(np.abs(ref_inv))
