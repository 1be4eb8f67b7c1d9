"""FP32 mixed form against the FP64 plain form (the oracle of the mixed form): the background
split (delta f = f - f0(u, v) in FP32, the RHS of f0 from FP64 tables) against the plain FP32
state, on configuration 1 (16^3 elements, n = 8, loss cone times 1 + 0.01 cos kx)."""
import numpy as np
import pytest

from helpers import history_err, rel_err

pytestmark = pytest.mark.gpu


def _run(precision, split=True, steps=200):
    from vlasov1d2v_b200 import problem
    from vlasov1d2v_b200.grid import Distribution

    if not split:
        orig = Distribution.__init__

        def init(self, *a, **kw):
            kw["background_split"] = False
            orig(self, *a, **kw)

        Distribution.__init__ = init
    try:
        p = problem.build((16, 16, 16), 8, perturbation="cos", amp=0.01, batch_steps=50,
                          precision=precision)
    finally:
        if not split:
            Distribution.__init__ = orig
    p.stepper.run_steps(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, steps)
    f = p.f.full_array().get() if precision == "fp32" else p.f.arr.get()
    return np.asarray(p.stepper.field_energy), f


def test_fp32_background_split_against_fp64(cuda):
    e64, f64 = _run("fp64")
    e32, f32 = _run("fp32")
    e32p, f32p = _run("fp32", split=False)
    err_split, err_plain = history_err(e32, e64), history_err(e32p, e64)
    ferr_split, ferr_plain = rel_err(f32, f64), rel_err(f32p, f64)
    print(f"energy history: split {err_split:.2e}, plain {err_plain:.2e}; "
          f"state: split {ferr_split:.2e}, plain {ferr_plain:.2e}")
    assert err_split < 1e-5
    assert ferr_split < 3e-6
    # the split removes the FP32 cancellation of the background in the x derivative
    assert ferr_split < ferr_plain / 4


@pytest.mark.parametrize("split", [True, False], ids=["background_split", "plain_fp32"])
def test_fp32_generic_tma_form_in_the_loop(cuda, split, monkeypatch):
    """FP32 order 6 on 16-byte rows, where the generic kernel's TMA form is the stage kernel (with
    the background split it stages the two background tables as 2-D boxes).  6 steps with and
    without the split match a run on the register-pencil kernel (VLASOV1D2V_STAGE_KERNEL=pencil)."""
    from vlasov1d2v_b200 import problem

    def run(tma):
        for var in ("VLASOV1D2V_STAGE_KERNEL", "VLASOV1D2V_GEN_NO_TMA"):
            monkeypatch.delenv(var, raising=False)
        if not tma:
            monkeypatch.setenv("VLASOV1D2V_STAGE_KERNEL", "pencil")
        p = problem.build((4, 4, 6), 6, perturbation="cos", amp=0.01, batch_steps=3, precision="fp32",
                          background_split=split)
        p.stepper.run_steps(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, 6)
        return np.asarray(p.stepper.field_energy), p.f.full_array().get()

    w0, f0 = run(False)
    w1, f1 = run(True)
    assert rel_err(f1, f0) < 1e-5
    assert history_err(w1, w0) < 1e-4
