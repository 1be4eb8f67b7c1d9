"""Parity on the geometries the benchmark times.

The benchmark grids (Nx = 32, Nu = Nv = 50, n = 8 and Nx = Nu = Nv = 64, n = 9) are too large for
the CPU oracle to step in seconds, but the stage kernels' tile and row geometry depends only on
the velocity grid and the order: an x-slab with the benchmark's own velocity grid runs the same
tiles (the ragged 4-element v tile at Nv = 50, the 66 n-wide rows at Nv = 64) through the same
kernel.  FP64 steps are held to the 1e-12 bar against the oracle; FP32 stages (plain and with
the background split) to FP32 rounding of the stage result.  The amplitude of the cos
perturbation is large so that the field keeps the relative rounding of the density.
"""
import numpy as np
import pytest
import torch

from helpers import F_RTOL, INNER, history_err, rel_err
from oracle import vlasov_oracle as vo

pytestmark = pytest.mark.gpu


def _oracle_steps(p, res, n, steps):
    c = vo.make_case(*res, n)
    f_host = p.f.arr.get().copy()
    rho = vo.moment_zero(f_host, c)
    E0, _ = vo.poisson2(rho - np.mean(rho), c)
    rec = vo.run(f_host, c, steps=steps, E0=E0)
    return f_host, rec


@pytest.mark.parametrize("res,n,steps", [((2, 50, 50), 8, 2), ((3, 50, 50), 8, 1), ((2, 64, 64), 9, 1)],
                         ids=["medium_slab_n8", "medium_slab3_n8", "large_slab_n9"])
def test_fp64_steps_on_benchmark_velocity_grids(cuda, res, n, steps):
    from vlasov1d2v_b200 import problem

    p = problem.build(res, n, perturbation="cos", amp=0.3, batch_steps=steps)
    f_ref, rec = _oracle_steps(p, res, n, steps)
    p.stepper.run_steps(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, steps)
    torch.cuda.synchronize()
    f = p.f.arr.get()
    assert rel_err(f[INNER], f_ref[INNER]) < F_RTOL
    np.testing.assert_allclose(p.stepper.field_energy, rec.field_energy, rtol=F_RTOL, atol=0)
    np.testing.assert_allclose(p.stepper.time_array, rec.time_array, rtol=1e-14, atol=0)


def _stage_check(ctx, c, n, res, seed, tol, bg=None):
    """The three RK stage kinds of a random FP32 state against the FP64 oracle."""
    from vlasov1d2v_b200 import _lib

    rng = np.random.default_rng(seed)
    fin = rng.standard_normal(c.shape).astype(np.float32).astype(np.float64)
    fin[0], fin[-1] = fin[-2], fin[1]  # periodic x ghosts: stage semantics
    fn = rng.standard_normal(c.shape).astype(np.float32).astype(np.float64)
    E = rng.standard_normal((res[0] + 2, n))
    R = vo.rhs(fin, E, c)
    if bg is not None:
        R = R + bg(E)
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
        err = rel_err(out.cpu().numpy().astype(np.float64)[INNER], want[INNER])
        assert err < tol, (stage, err)


@pytest.mark.parametrize("res,n", [((2, 50, 50), 8), ((2, 3, 5), 8), ((2, 4, 6), 4), ((2, 3, 5), 4),
                                   ((2, 64, 64), 9)],
                         ids=["medium_slab_n8", "ragged_n8", "n4_even", "n4_odd", "large_slab_n9"])
def test_fp32_stage_kernels_against_oracle(cuda, res, n):
    """FP32 stage kernels of the orders the generic FP32 test leaves out: n = 8 (the fragment
    kernel, full and ragged v tiles), n = 4 (the TMA kernel) and the large grid's n = 9 rows."""
    from vlasov1d2v_b200 import problem
    from vlasov1d2v_b200.context import get_context

    p = problem.build(res, n, perturbation=None, amp=0.0, precision="fp32", background_split=False)
    c = vo.make_case(*res, n)
    ctx = get_context(p.grids, precision="fp32", accel=p.refs.electron_acceleration_multiplier,
                      bfield=p.elliptic.magnetic_field, kappa=p.elliptic.poisson_coefficient,
                      courant=p.stepper.courant)
    ctx.set_background(None)
    _stage_check(ctx, c, n, res, 700 + n + res[2], 1e-5)


@pytest.mark.parametrize("res,n", [((2, 50, 50), 8), ((2, 64, 64), 9)], ids=["medium_slab_n8", "large_slab_n9"])
def test_fp32_background_split_steps_on_benchmark_velocity_grids(cuda, res, n):
    """The benchmarked FP32 mixed form (delta f in FP32, the background RHS from FP64 tables)
    over two steps against the FP64 oracle: f, and the energy history normwise."""
    from vlasov1d2v_b200 import problem

    p = problem.build(res, n, perturbation="cos", amp=0.3, batch_steps=2, precision="fp32")
    f_ref = None
    q = problem.build(res, n, perturbation="cos", amp=0.3, batch_steps=2)
    f_ref, rec = _oracle_steps(q, res, n, 2)
    p.stepper.run_steps(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, 2)
    torch.cuda.synchronize()
    f = p.f.full_array().get()
    assert rel_err(f[INNER], f_ref[INNER]) < 2e-6
    assert history_err(p.stepper.field_energy, rec.field_energy) < 1e-5


@pytest.mark.parametrize("res", [(2, 3, 5), (2, 50, 50)], ids=["ragged", "medium_slab"])
def test_fp32_n8_directional_rhs_against_oracle(cuda, res):
    """vl_rhs_weighted on the FP32 n = 8 kernel: the three single-direction RHS (x, u, v flux
    terms, each with its Jacobian as the weight and the other two weights zero) sum to the
    oracle's full RHS within FP32 rounding, and each of them is a non-trivial part of it."""
    from vlasov1d2v_b200 import _lib, problem
    from vlasov1d2v_b200.context import get_context

    n = 8
    p = problem.build(res, n, perturbation=None, amp=0.0, precision="fp32", background_split=False)
    c = vo.make_case(*res, n)
    ctx = get_context(p.grids, precision="fp32", accel=p.refs.electron_acceleration_multiplier,
                      bfield=p.elliptic.magnetic_field, kappa=p.elliptic.poisson_coefficient,
                      courant=p.stepper.courant)
    ctx.set_background(None)
    rng = np.random.default_rng(900 + res[2])
    f = rng.standard_normal(c.shape).astype(np.float32).astype(np.float64)
    E = rng.standard_normal((res[0] + 2, n))
    tf = torch.as_tensor(f, dtype=torch.float32, device="cuda")
    tE = torch.as_tensor(E, device="cuda")
    J = (c.x.J, c.u.J, c.v.J)
    parts = []
    for d in range(3):
        w = [0.0, 0.0, 0.0]
        w[d] = J[d]
        out = torch.zeros_like(tf)
        ctx.rhs_weighted(tf, tE, out, w, xhalo=_lib.VL_XHALO_GHOST)
        parts.append(out.cpu().numpy().astype(np.float64)[INNER])
    R = vo.rhs(f, E, c)[INNER]
    assert rel_err(parts[0] + parts[1] + parts[2], R) < 1e-5
    for part in parts:
        assert np.max(np.abs(part)) > 1e-3 * np.max(np.abs(R))
