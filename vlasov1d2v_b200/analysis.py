"""Run diagnostics on the host: growth rates of the field energy, history and state errors.

The field energy of a linearly unstable run grows as W(t) ~ exp(2 gamma t) once the fastest
mode dominates, so gamma is half the least-squares slope of ln W over that window.  These
helpers compare the mixed-precision form against the FP64 plain form on the same problem.
"""
import numpy as np


def growth_rate(time, energy, t0=None, t1=None):
    """Growth rate gamma of the field amplitude: half the least-squares slope of ln W(t) on
    [t0, t1] (the whole history when omitted).  Returns (gamma, rms residual of the fit)."""
    t = np.asarray(time, dtype=np.float64)
    w = np.asarray(energy, dtype=np.float64)
    m = np.isfinite(w) & (w > 0)
    if t0 is not None:
        m &= t >= t0
    if t1 is not None:
        m &= t <= t1
    if m.sum() < 3:
        raise ValueError("fewer than 3 samples in the fit window")
    tt, lw = t[m], np.log(w[m])
    a = np.vstack([tt, np.ones_like(tt)]).T
    coef, *_ = np.linalg.lstsq(a, lw, rcond=None)
    resid = lw - a @ coef
    return 0.5 * float(coef[0]), float(np.sqrt(np.mean(resid ** 2)))


def growth_window(time, energy, frac=0.25):
    """The window of relative width ``frac`` (of the history) whose ln W is closest to a
    straight line of positive slope: the phase of exponential growth.  Returns (t0, t1)."""
    t = np.asarray(time, dtype=np.float64)
    w = np.asarray(energy, dtype=np.float64)
    n = len(t)
    width = max(int(frac * n), 8)
    best, best_score = None, np.inf
    step = max(width // 8, 1)
    for s in range(0, n - width + 1, step):
        seg = slice(s, s + width)
        if np.any(w[seg] <= 0):
            continue
        g, r = growth_rate(t[seg], w[seg])
        if g <= 0:
            continue
        # residual relative to the growth over the window
        span = 2.0 * g * (t[s + width - 1] - t[s])
        score = r / span if span > 0 else np.inf
        if score < best_score:
            best, best_score = (float(t[s]), float(t[s + width - 1])), score
    if best is None:
        raise ValueError("no window of exponential growth found")
    return best


def history_error(a, b):
    """Normwise relative error of a history: max_t |a - b| / max_t |b|."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def state_errors(f, f_ref):
    """Max-norm and L2 relative errors of a state against a reference state."""
    f = np.asarray(f, dtype=np.float64)
    r = np.asarray(f_ref, dtype=np.float64)
    d = f - r
    return {"max_rel": float(np.max(np.abs(d)) / np.max(np.abs(r))),
            "l2_rel": float(np.linalg.norm(d.ravel()) / np.linalg.norm(r.ravel()))}
