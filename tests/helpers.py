"""Shared helpers of the test suite: golden fixtures, problem set-up, tolerances."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
INNER = (slice(1, -1), slice(None), slice(1, -1), slice(None), slice(1, -1), slice(None))
SMALL_CASES = ("tiny", "small", "n8", "n9")
EPS = np.finfo(np.float64).eps

# Parity bar of the FP64 plain form: f and field energy within 1e-12 relative of the reference.
F_RTOL = 1.0e-12


def golden(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.max(np.abs(b))
    if scale == 0:
        return float(np.max(np.abs(a)))
    return float(np.max(np.abs(a - b)) / scale)


def history_err(a, b):
    """Normwise relative error of a time history: max_t |a - b| / max_t |b|.  The field energy
    of the benchmark cases passes through deep minima (the field oscillates through zero), where
    a pointwise relative error is ill-conditioned for the reference itself."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def field_rtol(rho, base=F_RTOL):
    """Tolerance for fields derived from a density: E comes from rho - mean(rho), so rounding of
    rho (relative ~1e-16, summation-order dependent) is amplified by max|rho| / max|rho - mean|.
    The bar is ``base`` or 256 eps times that amplification, whichever is larger."""
    rho = np.asarray(rho)
    dev = np.max(np.abs(rho - rho.mean()))
    amp = np.max(np.abs(rho)) / dev if dev > 0 else 1.0
    return max(base, 256 * EPS * amp)


def case_setup(name):
    """Reference-normalised set-up of a golden case: returns (G, res, n, kwargs) for
    ``vlasov1d2v_b200.problem.build``."""
    G = golden(name)
    res = tuple(int(r) for r in G["res"])
    n = int(G["order"])
    return G, res, n
