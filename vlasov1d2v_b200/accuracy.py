"""Accuracy of the FP32 mixed form against the FP64 plain form on one problem.

    python -m vlasov1d2v_b200.accuracy --res 32 50 50 --order 8 --steps 2000

runs the same initial state (loss cone j = 6, 1e-3 cos kx + seeded 1e-6 noise per x node) in
both precisions on the GPU, and prints one JSON object: the field-energy growth rate of each
(least-squares fit of ln W over the detected window of exponential growth, the same window for
both), their relative difference, the normwise energy-history error, the final-state errors and
the wall time per step of each run.  The FP64 plain form matches the reference to 1e-12, so it
serves as the oracle for the mixed form.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def run(res, order, steps, precision, perturbation="cos", amp=1.0e-3, noise=1.0e-6, seed=0,
        batch=64, background_split=True):
    import torch

    from . import problem

    p = problem.build(tuple(res), order, perturbation=perturbation, amp=amp, noise=noise,
                      seed=seed, precision=precision, batch_steps=batch,
                      background_split=background_split)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    p.stepper.run_steps(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, steps)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    f = p.f.full_array().as_subclass(torch.Tensor)
    inner = f[1:-1, :, 1:-1, :, 1:-1, :].double().cpu().numpy()
    return {"time": np.asarray(p.stepper.time_array), "energy": np.asarray(p.stepper.field_energy),
            "f": inner, "wall_s": wall}


def compare(r64, r32, window=None):
    from .analysis import growth_rate, growth_window, history_error, state_errors

    t, w64, w32 = r64["time"], r64["energy"], r32["energy"]
    n = min(len(w64), len(w32))
    if window is None:
        window = growth_window(t[:n], w64[:n])
    g64, res64 = growth_rate(t[:n], w64[:n], *window)
    g32, res32 = growth_rate(r32["time"][:n], w32[:n], *window)
    return {
        "steps": n - 1,
        "final_time_fp64": float(t[n - 1]), "final_time_fp32": float(r32["time"][n - 1]),
        "growth_window": list(window),
        "growth_rate_fp64": g64, "growth_rate_fp32": g32,
        "growth_rate_rel_diff": abs(g32 - g64) / abs(g64),
        "fit_rms_residual_fp64": res64,
        "energy_history_err": history_error(w32[:n], w64[:n]),
        "energy_final_rel_err": abs(w32[n - 1] - w64[n - 1]) / abs(w64[n - 1]),
        "energy_growth_factor": float(w64[n - 1] / w64[0]),
        "state_err": state_errors(r32["f"], r64["f"]),
        "ms_per_step_fp64": 1e3 * r64["wall_s"] / (n - 1),
        "ms_per_step_fp32": 1e3 * r32["wall_s"] / (n - 1),
    }


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--res", type=int, nargs=3, default=[32, 50, 50])
    ap.add_argument("--order", type=int, default=8)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--window", type=float, nargs=2, default=None,
                    help="growth-rate fit window [t0, t1] (default: detected from the FP64 run)")
    ap.add_argument("--save", default=None, help="write both time/energy histories to this .npz")
    ap.add_argument("--perturbation", choices=("cos", "eigenmode"), default="cos",
                    help="cos: 1e-3 cos kx + 1e-6 noise; eigenmode: the reference's unstable "
                         "Bessel-series mode (om = -0.349i, delta_n = 1e-3)")
    ap.add_argument("--no-split", action="store_true",
                    help="FP32 run without the background split (plain FP32 state f)")
    args = ap.parse_args(argv)
    r64 = run(args.res, args.order, args.steps, "fp64", perturbation=args.perturbation)
    r32 = run(args.res, args.order, args.steps, "fp32", perturbation=args.perturbation,
              background_split=not args.no_split)
    if args.save:
        np.savez(args.save, time64=r64["time"], energy64=r64["energy"], time32=r32["time"],
                 energy32=r32["energy"])
    out = {"res": args.res, "order": args.order, "perturbation": args.perturbation,
           "fp32_background_split": not args.no_split}
    out.update(compare(r64, r32, tuple(args.window) if args.window else None))
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
