"""The allocation-free loop entry point against the regular one.

``vl_ssp_rk3_steps_noalloc`` serves callers that cannot allocate device memory (a host that
records into a CUDA graph while allocation is forbidden, a plugin whose framework owns the
device heap, a binding with nothing but raw pointers and a stream): the loop's moment scratch
is a fixed device array inside the library instead of a caller workspace.  Here the same
problem is advanced through both entry points, twice in a row, and the states, fields and
histories must agree within the FP64 parity bar of the suite.
"""
import numpy as np
import pytest
import torch

from helpers import F_RTOL, INNER, history_err, rel_err

pytestmark = pytest.mark.gpu


def _setup(res=(3, 4, 5), n=8):
    from vlasov1d2v_b200 import _lib, problem
    from vlasov1d2v_b200.context import get_context
    from vlasov1d2v_b200.timestep import _BIG_STEPS, _Run, get_max_speeds

    p = problem.build(res, n, perturbation="cos", amp=0.01)
    st = p.stepper
    st.adapt_time_step(get_max_speeds(p.grids, p.elliptic, p.refs), p.grids.x.dx, p.grids.u.dx,
                       p.grids.v.dx)
    ctx = get_context(p.grids, accel=p.refs.electron_acceleration_multiplier,
                      bfield=p.elliptic.magnetic_field, kappa=p.elliptic.poisson_coefficient,
                      courant=st.courant)
    # the fixed scratch holds this problem with room to spare (the rejection above the capacity
    # cannot be reached by the grids the kernels accept)
    assert 0 < ctx.workspace_bytes <= _lib.NOALLOC_SCRATCH_BYTES // 4
    runs = []
    for _ in range(2):
        f = p.f.arr.as_subclass(torch.Tensor).clone()
        run = _Run(ctx, f, hist_cap=8)
        run.sync_ghosts()
        run.upload_state(st._host_state(run, float("inf"), _BIG_STEPS))
        runs.append(run)
    return ctx, runs


def test_noalloc_loop_matches_workspace_loop(cuda):
    ctx, (ra, rb) = _setup()
    # a second problem of another size and order: its calls leave their own data in the shared
    # scratch (the moment partials of another grid and kernel layout)
    ctx2, (_, rc) = _setup((5, 3, 4), 4)
    for call in range(2):   # two calls in a row: the shared scratch carries the last call's data
        ctx.ssp_rk3_steps(ra.f, ra.sa, ra.sb, ra.E, ra.phi, ra.state, 3)
        ctx.ssp_rk3_steps_noalloc(rb.f, rb.sa, rb.sb, rb.E, rb.phi, rb.state, 3)
        ctx2.ssp_rk3_steps_noalloc(rc.f, rc.sa, rc.sb, rc.E, rc.phi, rc.state, 2)
        torch.cuda.synchronize()
        sa, sb = ra.read_state(), rb.read_state()
        assert sa.status == 0 and sb.status == 0 and rc.read_state().status == 0
        assert sa.steps == sb.steps == 3 * (call + 1)
        fa = ra.f.cpu().numpy()
        fb = rb.f.cpu().numpy()
        assert rel_err(fb[INNER], fa[INNER]) <= F_RTOL
        assert rel_err(rb.E.cpu().numpy(), ra.E.cpu().numpy()) <= F_RTOL
        ha = ra.hist[:, :sa.steps].cpu().numpy()
        hb = rb.hist[:, :sb.steps].cpu().numpy()
        assert history_err(hb[0], ha[0]) <= F_RTOL
        np.testing.assert_allclose(hb[1:], ha[1:], rtol=F_RTOL)
