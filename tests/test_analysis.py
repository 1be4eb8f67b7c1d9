"""Host diagnostics: growth-rate fit and window detection on synthetic histories."""
import numpy as np

from vlasov1d2v_b200.analysis import growth_rate, growth_window, history_error, state_errors


def test_growth_rate_recovers_exponential():
    t = np.linspace(0.0, 50.0, 2001)
    w = 3e-9 * np.exp(2 * 0.0731 * t)
    g, r = growth_rate(t, w)
    assert abs(g - 0.0731) < 1e-12 and r < 1e-12


def test_growth_window_skips_transient_and_saturation():
    rng = np.random.default_rng(1)
    t = np.linspace(0.0, 100.0, 4001)
    lw = np.where(t < 20, -20 + 0.5 * np.sin(3 * t),            # oscillating transient
                  np.where(t < 70, -20 + 2 * 0.11 * (t - 20),   # linear growth
                           -20 + 2 * 0.11 * 50))                # saturation
    w = np.exp(lw + 1e-6 * rng.standard_normal(t.size))
    t0, t1 = growth_window(t, w, frac=0.2)
    assert 20 <= t0 and t1 <= 70
    g, _ = growth_rate(t, w, t0, t1)
    assert abs(g - 0.11) / 0.11 < 1e-4


def test_errors():
    a = np.array([1.0, 2.0, 4.0])
    assert history_error(a * (1 + 1e-9), a) < 2e-9
    e = state_errors(a + 1e-3, a)
    assert abs(e["max_rel"] - 2.5e-4) < 1e-12
