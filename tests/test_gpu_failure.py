"""Failure detection of the device loop: non-finite values injected into host-made inputs.

The loop's field solve flags a non-finite field, energy or dt in bit 0 of the loop state's
status word (``vl_run_state.status``); ``Stepper`` raises ``NonFiniteError`` when it reads it.
The reference's counterpart is a NaN check that is commented out in its time loop.  Each case
injects the value on the host (into the initial state or into the initial field), checks the
flag and the exception, and then runs a clean problem on the same device against the reference's
fixture: a detected failure leaves the GPU usable.  Nothing here faults or hangs the GPU.
"""
import numpy as np
import pytest
import torch

from helpers import F_RTOL, INNER, golden, rel_err

pytestmark = pytest.mark.gpu


def _clean_run_still_matches():
    from vlasov1d2v_b200 import problem

    G = golden("tiny_p")
    p = problem.build(tuple(int(r) for r in G["res"]), int(G["order"]), amp=float(G["delta_n"]))
    nst = len(G["energy"]) - 1
    p.stepper.run_steps(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, nst)
    np.testing.assert_allclose(p.stepper.field_energy, G["energy"], rtol=F_RTOL, atol=0)
    assert rel_err(p.f.arr.get()[INNER], G[f"f_step{nst}"]) < F_RTOL


def _poison_state(p, value, precision):
    """Host-made initial state with one interior node replaced by ``value``."""
    f = p.f.arr.get().copy() if precision == "fp64" else p.f.full_array().get().copy()
    f[2, 1, 2, 3, 3, 0] = value
    p.f.set_array(f)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("value", [np.nan, np.inf], ids=["nan", "inf"])
def test_nonfinite_state_raises_and_gpu_stays_usable(cuda, precision, value):
    from vlasov1d2v_b200 import problem
    from vlasov1d2v_b200.timestep import NonFiniteError

    p = problem.build((3, 4, 5), 4, perturbation="cos", amp=0.05, precision=precision,
                      final_time=1.0e9, batch_steps=4)
    _poison_state(p, value, precision)
    with pytest.raises(NonFiniteError):
        p.stepper.main_loop(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, None)
    # the flag is raised by the first step's field solve; the loop stops in that batch
    assert p.stepper.steps_counter <= 4
    torch.cuda.synchronize()
    _clean_run_still_matches()


def test_nonfinite_field_raises(cuda):
    """A non-finite initial field (host-made E): the initial dt is then NaN, the first stage
    spreads it into the state and the first field solve flags it."""
    from vlasov1d2v_b200 import problem
    from vlasov1d2v_b200.timestep import NonFiniteError

    p = problem.build((3, 4, 5), 4, perturbation="cos", amp=0.05, final_time=1.0e9, batch_steps=4)
    E = p.elliptic.electric_field.get().copy()
    E[2, 1] = np.nan
    p.elliptic.electric_field = torch.as_tensor(E, device="cuda")
    with pytest.raises(NonFiniteError):
        p.stepper.main_loop(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, None)
    _clean_run_still_matches()


def test_run_state_init_flags_nonfinite_field(cuda):
    """Through the C ABI: vl_run_state_init with a non-finite E0 sets status bit 0 and clears
    active_next, and a following vl_ssp_rk3_steps call takes no step and leaves f untouched."""
    from vlasov1d2v_b200 import _lib, problem
    from vlasov1d2v_b200.context import get_context
    from vlasov1d2v_b200.timestep import _Run

    p = problem.build((3, 4, 5), 4, perturbation="cos", amp=0.05)
    st = p.stepper
    ctx = get_context(p.grids, accel=p.refs.electron_acceleration_multiplier,
                      bfield=p.elliptic.magnetic_field, kappa=p.elliptic.poisson_coefficient,
                      courant=st.courant)
    f = p.f.arr.as_subclass(torch.Tensor).clone()
    run = _Run(ctx, f, hist_cap=8)
    run.sync_ghosts()
    E0 = p.elliptic.electric_field.as_subclass(torch.Tensor).clone()
    E0[1, 0] = float("inf")
    ctx.run_state_init(run.state, E0, 1.0e9, 100, run.hist[0], run.hist[1], run.hist[2])
    f_before = f.clone()
    ctx.ssp_rk3_steps(run.f, run.sa, run.sb, run.E, run.phi, run.state, 3)
    torch.cuda.synchronize()
    s = run.read_state()
    assert s.status & 1
    assert s.active_next == 0 and s.steps == 0
    assert torch.equal(f, f_before)
    assert _lib.VlRunState.from_buffer_copy(bytes(s)).status == s.status
    _clean_run_still_matches()
