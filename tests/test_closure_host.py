"""Host side of the learned closure: the fine -> coarse L2 projection matrices."""
import numpy as np

from vlasov1d2v_b200.basis import Basis1D
from vlasov1d2v_b200.closure import projection_1d


def test_projection_reproduces_coarse_polynomials():
    fine, coarse = Basis1D(8), Basis1D(6)
    xf, xc = np.asarray(fine.nodes, dtype=float), np.asarray(coarse.nodes, dtype=float)
    for ratio in (1, 3):
        P = projection_1d(xf, xc, ratio)
        # fine nodal values of a degree-5 polynomial on the ratio sub-elements
        poly = np.polynomial.Polynomial([0.3, -1.0, 0.5, 2.0, -0.7, 0.25])
        sub = np.concatenate([(-1 + (2 * q + 1) / ratio) + xf / ratio for q in range(ratio)])
        np.testing.assert_allclose(P @ poly(sub), poly(xc), rtol=0, atol=1e-12)


def test_projection_is_l2_orthogonal():
    fine, coarse = Basis1D(8), Basis1D(6)
    xf, xc = np.asarray(fine.nodes, dtype=float), np.asarray(coarse.nodes, dtype=float)
    P = projection_1d(xf, xc, 3)
    # a degree-7 piecewise function minus its projection is orthogonal to degree <= 5
    rng = np.random.default_rng(2)
    vals = rng.normal(size=24)
    proj = P @ vals
    xq, wq = np.polynomial.legendre.leggauss(30)
    from scipy.interpolate import lagrange

    pc = lagrange(xc, proj)
    for s in range(6):
        tot = 0.0
        for q in range(3):
            lo, hi = -1 + 2 * q / 3, -1 + 2 * (q + 1) / 3
            x = 0.5 * (hi - lo) * xq + 0.5 * (hi + lo)
            pf = lagrange(xf, vals[8 * q:8 * q + 8])
            tot += 0.5 * (hi - lo) * np.sum(wq * (pf(xq) - pc(x)) * np.polynomial.legendre.Legendre.basis(s)(x))
        assert abs(tot) < 1e-9


def test_runaway_criterion_ignores_oscillation_minima():
    """The closure loop's fallback test: field energy that oscillates through deep minima (plasma
    oscillation early in a run) or grows at a physical rate is not a runaway; energy shooting
    above its earlier maximum far faster than exp(2 max_rate t) is."""
    import math

    from vlasov1d2v_b200.closure import runaway

    t = [0.01 * i for i in range(400)]
    # cos^2 oscillation (deep minima) under slow physical growth (rate 0.05)
    w = [1e-6 * math.cos(3.0 * x) ** 2 * math.exp(2 * 0.05 * x) + 1e-14 for x in t]
    for start in range(50, 400, 50):   # every batch boundary, minima included
        assert not runaway(t[:start + 50], w[:start + 50], start, 0.5)
    # a batch that starts at a minimum and climbs back to the earlier peak is still physical
    i_min = min(range(100, 150), key=w.__getitem__)
    assert not runaway(t[:i_min + 60], w[:i_min + 60], i_min, 0.5)
    # runaway: a factor 1e3 above the earlier maximum within 0.5 time units
    bad = w[:200] + [max(w[:200]) * 1e3] * 50
    assert runaway(t[:250], bad, 200, 0.5)
