"""Batched heterogeneous ensemble: each member matches the same problem run alone."""
import numpy as np
import pytest

from helpers import history_err, rel_err

pytestmark = pytest.mark.gpu

MEMBERS = [
    dict(res=(3, 4, 5), order=3, om_pc=10.0, k=0.886, perturbation="cos", amp=0.02),
    dict(res=(4, 6, 5), order=4, om_pc=8.0, k=1.2, perturbation="eigenmode", amp=1e-2),
    dict(res=(2, 3, 4), order=8, om_pc=12.0, k=0.7, perturbation="cos", amp=0.01),
    dict(res=(3, 2, 3), order=6, om_pc=6.0, k=1.5, perturbation="cos", amp=0.005),
    dict(res=(2, 2, 2), order=9, om_pc=10.0, k=0.886, perturbation="cos", amp=0.01),
]


def _build(q, precision, batch):
    from vlasov1d2v_b200 import problem

    q = dict(q)
    return problem.build(q.pop("res"), q.pop("order"), precision=precision, batch_steps=batch,
                         background_split=False, **q)


@pytest.mark.parametrize("schedule", [(128, 2, 2), (0, 0, 2), (0, 1 << 8, 2), (0, 0x3FE, 2), (0, 0xFFFFFFFF, 2)],
                         ids=["fused", "by_order", "by_order_native8", "all_native", "native_auto"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-5)])
def test_ensemble_members_match_single_runs(cuda, precision, tol, schedule):
    from vlasov1d2v_b200.ensemble import Ensemble

    singles = []
    for q in MEMBERS:
        p = _build(q, precision, 3)
        for _ in range(2):
            p.stepper.run_steps(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, 3)
        singles.append(p)
    probs = [_build(q, precision, 3) for q in MEMBERS]
    ens = Ensemble(probs, batch_steps=3)
    ens.set_schedule(*schedule)
    ens.run_steps(3)
    ens.run_steps(3, use_graph=False)
    for p, s in zip(probs, singles):
        assert p.stepper.steps_counter == s.stepper.steps_counter == 6
        assert rel_err(p.f.arr.get(), s.f.arr.get()) < tol
        assert history_err(p.stepper.field_energy, s.stepper.field_energy) < tol
        np.testing.assert_allclose(p.stepper.time_array, s.stepper.time_array, rtol=tol)


@pytest.mark.parametrize("schedule", [None, (0, 0, 2), (0, 1 << 8, 2)], ids=["tuned", "by_order", "native8"])
def test_ensemble_final_times_and_autotune(cuda, schedule):
    from vlasov1d2v_b200.ensemble import Ensemble

    probs = [_build(q, "fp64", 8) for q in MEMBERS[:3]]
    dt0 = []
    for p in probs:
        from vlasov1d2v_b200.timestep import get_max_speeds

        p.stepper.adapt_time_step(get_max_speeds(p.grids, p.elliptic, p.refs), p.grids.x.dx,
                                  p.grids.u.dx, p.grids.v.dx)
        dt0.append(p.stepper.dt)
    # member 1 stops after about 2 steps, the others run the whole batch
    finals = [1e9, 2.5 * dt0[1], 1e9]
    ens = Ensemble(probs, final_time=finals, batch_steps=8)
    f_before = [p.f.arr.get().copy() for p in probs]
    cands = [(128, 1, 1), (128, 2, 2), (64, 2, 4), (0, 0, 4)]
    res = ens.autotune(candidates=cands, steps=2, cache_path=None)
    assert res["schedule"] in [list(c) for c in cands] and len(res["trials"]) == 4
    for p, f0 in zip(probs, f_before):   # tuning restored the states
        np.testing.assert_array_equal(p.f.arr.get(), f0)
    if schedule is not None:
        ens.set_schedule(*schedule)
    ens.run_steps(8)
    assert probs[0].stepper.steps_counter == 8 and probs[2].stepper.steps_counter == 8
    assert 2 <= probs[1].stepper.steps_counter <= 3
    assert probs[1].stepper.time >= finals[1]


@pytest.mark.parametrize("schedule", [(0, 0, 2), (0, 0xFFFFFFFF, 2), (128, 2, 2)],
                         ids=["by_order", "native_auto", "fused"])
def test_ensemble_members_against_oracle(cuda, schedule):
    """Every member (orders 3, 4, 6, 8, 9, each with its own grid and physics) stepped by the
    ensemble in FP64 against the CPU oracle run from the same initial state: f within 1e-12
    relative, the energy history within 1e-12 normwise and the clock within 1e-13."""
    from oracle import vlasov_oracle as vo
    from vlasov1d2v_b200.ensemble import Ensemble

    probs = [_build(q, "fp64", 3) for q in MEMBERS]
    refs = []
    for q, p in zip(MEMBERS, probs):
        res, n = q["res"], q["order"]
        c = vo.make_case(*res, n, om_pc=q["om_pc"], k=q["k"])
        f = p.f.arr.get().copy()
        rho = vo.moment_zero(f, c)
        E0, _ = vo.poisson2(rho - np.mean(rho), c)
        refs.append((f, vo.run(f, c, steps=3, E0=E0)))
    ens = Ensemble(probs, batch_steps=3)
    ens.set_schedule(*schedule)
    ens.run_steps(3)
    inner = (slice(1, -1), slice(None)) * 3
    for p, (f, rec) in zip(probs, refs):
        assert p.stepper.steps_counter == 3
        assert rel_err(p.f.arr.get()[inner], f[inner]) < 1e-12
        assert history_err(p.stepper.field_energy, rec.field_energy) < 1e-12
        np.testing.assert_allclose(p.stepper.time_array, rec.time_array, rtol=1e-13)
