"""The product's host-side set-up (basis, grids, DFT tables, normalisation, initial states) is
bit-identical to the reference's (fixtures in tests/golden).  No GPU needed."""
import numpy as np
import pytest

from helpers import SMALL_CASES, case_setup, golden
from vlasov1d2v_b200 import problem
from vlasov1d2v_b200.basis import Basis1D, Basis3D
from vlasov1d2v_b200.grid import Distribution, Grid3D
from vlasov1d2v_b200.timestep import Stepper, courant_numbers


@pytest.mark.parametrize("n", range(1, 11))
def test_basis_bit_identical(n):
    g = golden("basis")
    b = Basis1D(n)
    np.testing.assert_array_equal(np.asarray(b.nodes, dtype=float), g[f"n{n}_nodes"])
    np.testing.assert_array_equal(np.asarray(b.weights, dtype=float), g[f"n{n}_weights"])
    np.testing.assert_array_equal(b.vandermonde_inverse, g[f"n{n}_vinv"])
    np.testing.assert_array_equal(b.invm, g[f"n{n}_invm"])
    np.testing.assert_array_equal(b.np_up, g[f"n{n}_up"])
    np.testing.assert_array_equal(b.np_xi, g[f"n{n}_xi"])


def test_courant_table():
    np.testing.assert_array_equal(courant_numbers[3], golden("basis")["courant_rk3"])
    assert Stepper(3, 8, 1.0, 1.0).courant == 0.040
    with pytest.raises(IndexError):  # the reference's table has 9 entries (n = 10 fails too)
        Stepper(3, 10, 1.0, 1.0)


@pytest.mark.parametrize("name", SMALL_CASES)
def test_grids_bit_identical(name):
    G, res, n = case_setup(name)
    basis = Basis3D(np.array([n] * 3))
    grids = Grid3D(basis, G["lows"], G["highs"], np.array(res))
    np.testing.assert_array_equal(grids.x.arr, G["x_arr"])
    np.testing.assert_array_equal(grids.u.arr, G["u_arr"])
    np.testing.assert_array_equal(grids.v.arr, G["v_arr"])
    np.testing.assert_array_equal(grids.x.wave_numbers, G["wave_numbers"])
    np.testing.assert_array_equal(grids.x.np_spectral_transform, G["T"])
    np.testing.assert_array_equal(grids.x.np_grid_phases, G["P"])
    # the factored tables the native field solve reads: T = phase ell exactly as the reference
    # forms it, and the inverse phases conj(phase) qnode within rounding of the coordinates
    x = grids.x
    T = np.transpose(x.np_dft_phase[:, :, None] * x.np_dft_ell.T[None, :, :], (0, 2, 1))
    np.testing.assert_array_equal(T, G["T"])
    P = np.conj(x.np_dft_phase).T[:, :, None] * x.np_dft_qnode.T[:, None, :]
    assert np.max(np.abs(P - G["P"])) < 1e-13


@pytest.mark.parametrize("name", SMALL_CASES)
def test_initial_state_bit_identical(name):
    G, res, n = case_setup(name)
    refs = problem.default_reference()
    basis = Basis3D(np.array([n] * 3))
    grids = Grid3D(basis, G["lows"], G["highs"], np.array(res))
    d = Distribution(vt=refs.vt_e, ring_j=6, resolutions=res, orders=[n] * 3, om=-0.349j,
                     om_pc=10.0, delta_n=1e-3)
    np.testing.assert_array_equal(d.initial_array(grids), G["f_init"])


def test_normalisation_bit_identical():
    G = golden("tiny")
    refs = problem.default_reference()
    assert refs.electron_acceleration_multiplier == G["accel"]
    assert refs.charge_density_multiplier == G["kappa"]
    assert (refs.omp_e_tau / refs.omc_e_tau) / 10.0 == G["B"]
    assert refs.vt_e == G["vt"]


def test_cfg1_initial_state():
    G = golden("cfg1_200")
    refs = problem.default_reference()
    basis = Basis3D(np.array([8] * 3))
    L = 2 * np.pi / (0.886 / 10.0)
    vm = 8.5 * refs.vt_e
    grids = Grid3D(basis, np.array([-L / 2, -vm, -vm]), np.array([L / 2, vm, vm]),
                   np.array([16, 16, 16]))
    f = problem.cos_perturbed(grids, refs.vt_e, 6, 0.01)
    assert f.sum() == G["f_init_sum"]
    np.testing.assert_array_equal(f[5, 3, 7, 2, 9, 4:8], G["f_init_probe"])
