"""The reference's driver script, ``main/main.py``, run unchanged on this package.

The script is not part of this repository: set ``VLASOV_REFERENCE_MAIN`` to the reference
checkout's ``main/`` directory to run these tests (they skip without it).  The CPU test checks
that every name the script imports or calls on ``cupy`` resolves; the GPU test executes the
script (4 x 40 x 40 elements, order 8, eigenmode perturbation, to t = 2) through
``vlasov1d2v_b200.reference_driver`` and compares its first steps with the oracle and its whole
field-energy history with the same problem built through ``problem.build``.
"""
import ast
import os

import numpy as np
import pytest

REF_MAIN = os.environ.get("VLASOV_REFERENCE_MAIN", "")
SCRIPT = os.path.join(REF_MAIN, "main.py") if REF_MAIN else ""
needs_script = pytest.mark.skipif(not (SCRIPT and os.path.isfile(SCRIPT)),
                                  reason="VLASOV_REFERENCE_MAIN does not name the reference's main/ directory")


@needs_script
def test_driver_names_resolve():
    from vlasov1d2v_b200 import cupy_compat, reference_driver

    tree = ast.parse(open(SCRIPT).read())
    imported = set()
    cp_calls = set()
    for node in ast.walk(tree):
        if isinstance(node, ast.Import):
            imported.update(a.name for a in node.names)
        if isinstance(node, ast.Attribute) and isinstance(node.value, ast.Name) and node.value.id == "cp":
            cp_calls.add(node.attr)
    missing = [c for c in cp_calls if not hasattr(cupy_compat, c)]
    assert not missing, missing
    known = set(reference_driver._ALIASES) | {"numpy", "cupy", "matplotlib", "matplotlib.pyplot", "pyvista"}
    assert imported <= known, imported - known


@needs_script
@pytest.mark.gpu
def test_driver_runs_unchanged(cuda, tmp_path):
    import torch

    from oracle import vlasov_oracle as vo
    from vlasov1d2v_b200 import problem
    from vlasov1d2v_b200.reference_driver import run_driver

    g = run_driver(SCRIPT, workdir=str(tmp_path))
    st, f0 = g["stepper"], g["f0"]
    res = tuple(int(r) for r in g["resolutions"])
    n = int(g["order"])
    assert st.time >= float(g["final_time"]) and st.steps_counter > 10
    # the same problem through the package's own builder and loop
    p = problem.build(res, n, om_pc=float(g["om_pc"]), ring_j=int(g["ring_j"]), amp=float(g["delta_n"]),
                      final_time=float(g["final_time"]), write_time=float(g["write_time"]))
    f_init = p.f.arr.get().copy()
    p.stepper.main_loop(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, None)
    torch.cuda.synchronize()
    assert p.stepper.steps_counter == st.steps_counter
    np.testing.assert_array_equal(np.asarray(st.field_energy), np.asarray(p.stepper.field_energy))
    np.testing.assert_array_equal(f0.arr.get(), p.f.arr.get())
    # the first steps against the oracle (the density-cancellation-aware bar of the suite: the
    # driver's 1e-3 perturbation amplifies the density's rounding into the field)
    from helpers import field_rtol

    c = vo.make_case(*res, n)
    rho = vo.moment_zero(f_init, c)
    E0, _ = vo.poisson2(rho - np.mean(rho), c)
    rec = vo.run(f_init, c, steps=3, E0=E0)
    np.testing.assert_allclose(st.field_energy[:4], rec.field_energy, rtol=2 * field_rtol(rho), atol=0)
    np.testing.assert_allclose(st.time_array[:4], rec.time_array, rtol=1e-13)
    # the run files the script asked for exist
    assert any(name.endswith("_info.txt") for name in os.listdir(tmp_path))
