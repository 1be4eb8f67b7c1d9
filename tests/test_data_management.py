"""Run output and checkpoints: the reference's dataset layout, info-file round trip (host)."""
from types import SimpleNamespace

import numpy as np

from vlasov1d2v_b200 import data_management as dm
from vlasov1d2v_b200 import problem


def _geo():
    return np.array([[-35.0, 35.0, 4, 8], [-8.5, 8.5, 6, 8], [-8.5, 8.5, 5, 8]])


def test_run_file_round_trip(tmp_path):
    refs = problem.default_reference()
    shape = (6, 8, 8, 8, 7, 8)
    folder = str(tmp_path) + "/"
    rd = dm.RunData(folder, "run", shape, _geo(), np.array([10.0, 0.5, 0.04, 3]), refs)
    rng = np.random.default_rng(0)
    snaps = []
    for s in range(3):
        f = rng.standard_normal(shape)
        el = SimpleNamespace(potential=rng.standard_normal((4, 8)))
        dens = rng.standard_normal((4, 8))
        if s == 0:
            rd.create_file(f, el, dens)
            snaps.append((0.0, f, el.potential, dens, 0.0))
        else:
            rd.save_data(f, el, dens, time=0.1 * s, field_energy=1e-3 * s)
            snaps.append((0.1 * s, f, el.potential, dens, 1e-3 * s))
    rr = dm.ReadData(folder, "run")
    t, pdf, pot, den, eng = rr.read_data()
    assert pdf.shape == (3, *shape) and pdf.dtype == np.float32
    for k, (ts, f, p, d, e) in enumerate(snaps):
        assert t[k] == ts and eng[k] == e
        np.testing.assert_array_equal(pdf[k], f.astype(np.float32))
        np.testing.assert_array_equal(pot[k], p.astype(np.float32))
        np.testing.assert_array_equal(den[k], d.astype(np.float32))
    t1, pdf1, pot1 = rr.read_specific_time(1)
    np.testing.assert_array_equal(pdf1, snaps[1][1].astype(np.float32))
    tr, pr = rr.read_potential_only((1, 3))
    assert len(tr) == 2 and pr.shape == (2, 4, 8)
    orders, resolutions, lows, highs, time_info, ref_values = rr.read_info()
    assert list(orders) == [8, 8, 8] and list(resolutions) == [4, 6, 5]
    assert lows[0] == -35.0 and highs[0] == 35.0 and time_info[0] == 10.0
