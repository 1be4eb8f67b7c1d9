"""The closure MLP's CPU oracle: its backward pass against finite differences (FP64, no bf16
rounding), so that it can serve as the oracle of the GPU kernels."""
import numpy as np

from oracle import mlp_oracle as mo


def _params(rng):
    W = [rng.normal(0, np.sqrt(2.0 / k), size=(k, n)) for k, n in mo.DIMS]
    b = [rng.normal(0, 0.1, size=n) for _, n in mo.DIMS]
    return W, b


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    W, b = _params(rng)
    X = rng.normal(size=(5, mo.IN))
    T = rng.normal(size=(5, mo.OUT))
    nout = 36
    Y, H, Z = mo.forward(X, W, b, round_bf16=False)
    dW, db = mo.backward(Y, T, W, H, Z, nout, round_bf16=False)
    h = 1e-6
    for l, (i, j) in [(0, (3, 7)), (1, (5, 9)), (2, (0, 127)), (3, (11, 30))]:
        Wp = [w.copy() for w in W]
        Wp[l][i, j] += h
        Wm = [w.copy() for w in W]
        Wm[l][i, j] -= h
        lp = mo.loss(mo.forward(X, Wp, b, False)[0], T, nout)
        lm = mo.loss(mo.forward(X, Wm, b, False)[0], T, nout)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - dW[l][i, j]) <= 1e-6 * max(1.0, abs(fd)), (l, fd, dW[l][i, j])
    bp = [v.copy() for v in b]
    bp[1][4] += h
    bm = [v.copy() for v in b]
    bm[1][4] -= h
    fd = (mo.loss(mo.forward(X, W, bp, False)[0], T, nout) - mo.loss(mo.forward(X, W, bm, False)[0], T, nout)) / (2 * h)
    assert abs(fd - db[1][4]) <= 1e-6 * max(1.0, abs(fd))


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159265, 1e-20], dtype=np.float64)
    r = mo.bf16(x)
    # 8 significant bits: 1 + 2^-8 is a tie between 1 and 1 + 2^-7 -> even (1.0)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12
