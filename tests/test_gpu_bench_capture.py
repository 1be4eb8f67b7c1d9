"""The benchmark's captured K-step graph replays the same steps as the Stepper's own launches: for
the FP32 mixed form (background split) the captured stage kernels must carry the background RHS
tables.  Two steps from the same initial state, bench.capture_steps + replay against
run.launch, states and loop histories equal."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("res,order", [((4, 6, 6), 8), ((2, 4, 4), 9)])
def test_bench_graph_matches_stepper_launch(cuda, res, order):
    import bench
    from vlasov1d2v_b200 import problem
    from vlasov1d2v_b200.timestep import _BIG_STEPS, get_max_speeds

    p = problem.build(res, order, perturbation="cos", amp=1.0e-3, noise=1.0e-6, seed=0,
                      precision="fp32", batch_steps=2)
    assert p.f.background_split
    st = p.stepper
    st.adapt_time_step(max_speeds=get_max_speeds(p.grids, p.elliptic, p.refs),
                       dx=p.grids.x.dx, du=p.grids.u.dx, dv=p.grids.v.dx)
    run = st._run(p.f, p.elliptic, p.grids, p.refs)
    assert run.background is not None
    host_state = st._host_state(run, float("inf"), _BIG_STEPS)
    f0 = run.f.clone()

    run.upload_state(host_state)
    run.launch(2, use_graph=False)
    torch.cuda.synchronize()
    want_f = run.f.clone()
    want_h = run.hist[:, :2].clone()

    run.f.copy_(f0)
    run.upload_state(host_state)
    g = bench.capture_steps(run, 2)
    run.f.copy_(f0)
    run.upload_state(host_state)
    g.replay()
    torch.cuda.synchronize()
    assert run.read_state().status == 0
    np.testing.assert_array_equal(run.f.cpu().numpy(), want_f.cpu().numpy())
    np.testing.assert_array_equal(run.hist[:, :2].cpu().numpy(), want_h.cpu().numpy())
    del g
