"""The learned-closure experiment: train on fine runs, evaluate on a held-out fine run.

    python -m vlasov1d2v_b200.closure_experiment [--draws 4] [--snapshots 8] [--every 25]

Fine runs (Nx = 16, Nu = Nv = 60, order 8, FP64) of seeded parameter draws from the batched
benchmark's distribution (k ~ U[0.5, 2], loss-cone index j in {3..6}, omega_p / omega_c ~
U[5, 15], amplitude log-U[1e-4, 1e-2], cos kx perturbation) give training pairs on the coarse
grid (Nx = 16, Nu = Nv = 20, order 6): features of the projected fine state and the RHS
correction P R_fine - R_coarse.  The network is trained on the GPU with the project's kernels.
A held-out draw is then run three ways to a common final time -- fine, plain coarse and coarse
with the closure -- and the field-energy growth rate, the final-state L2 error (against the
projected fine state) and the device time of each run are reported as one JSON object.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch


def _log(rec):
    import sys

    print(json.dumps(rec), file=sys.stderr, flush=True)


def _draws(count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        out.append({"k": float(rng.uniform(0.5, 2.0)), "ring_j": int(rng.choice([3, 4, 5, 6])),
                    "om_pc": float(rng.uniform(5.0, 15.0)), "amp": float(10 ** rng.uniform(-4.0, -2.0))})
    return out


def _problems(q, fine_res, coarse_res):
    from . import problem

    kw = dict(k=q["k"], ring_j=q["ring_j"], om_pc=q["om_pc"], perturbation="cos", amp=q["amp"])
    fine = problem.build(fine_res, 8, batch_steps=50, **kw)
    coarse = problem.build(coarse_res, 6, batch_steps=50, **kw)
    return fine, coarse


def _timed(fn):
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fn()
    torch.cuda.synchronize()
    return time.perf_counter() - t0


def _run_to(p, t_end, batch=50):
    st = p.stepper
    st.final_time = t_end
    st.batch_steps = batch
    st.verbose = False
    st.main_loop(p.f, p.basis, p.elliptic, p.grids, p.flux, p.refs, None)


def main(argv=None):
    from .basis import Basis1D
    from .closure import MLP, ClosureStepper, Projector, evaluate, make_pair, train
    from .analysis import growth_rate, growth_window

    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--draws", type=int, default=4)
    ap.add_argument("--snapshots", type=int, default=8)
    ap.add_argument("--every", type=int, default=25)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--t-end", type=float, default=30.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--noise", type=float, default=0.02, help="feature noise during training")
    ap.add_argument("--fine-res", type=int, nargs=3, default=[16, 60, 60])
    ap.add_argument("--coarse-res", type=int, nargs=3, default=[16, 20, 20])
    ap.add_argument("--alpha", type=float, nargs="+", default=[1.0],
                    help="scales of the learned correction to run (1: as trained)")
    ap.add_argument("--constraint", nargs="+", default=["none"], choices=["none", "charge"],
                    help="forms of the correction to run: as predicted, or charge-conserving")
    args = ap.parse_args(argv)
    fine_res, coarse_res = tuple(args.fine_res), tuple(args.coarse_res)
    escale = 0.05
    proj = Projector(np.asarray(Basis1D(8).nodes, float), np.asarray(Basis1D(6).nodes, float),
                     fine_res[1] // coarse_res[1])
    out = {"fine_res": fine_res, "coarse_res": coarse_res}
    # ---- training data ----
    t0 = time.perf_counter()
    Xs, Ts = [], []
    draws = _draws(args.draws + 1, args.seed)
    for q in draws[:-1]:
        fine, coarse = _problems(q, fine_res, coarse_res)
        for _ in range(args.snapshots):
            fine.stepper.run_steps(fine.f, fine.basis, fine.elliptic, fine.grids, fine.flux, fine.refs,
                                   args.every)
            X, T = make_pair(fine, coarse, proj, escale)
            Xs.append(X)
            Ts.append(T)
        del fine, coarse
    X, T = torch.cat(Xs), torch.cat(Ts)
    del Xs, Ts
    n = X.shape[0]
    perm = torch.randperm(n, device=X.device, generator=torch.Generator(device=X.device).manual_seed(1))
    nval = n // 20
    Xv, Tv = X[perm[:nval]].contiguous(), T[perm[:nval]].contiguous()
    Xt, Tt = X[perm[nval:]].contiguous(), T[perm[nval:]].contiguous()
    out["samples"] = int(n)
    out["data_s"] = time.perf_counter() - t0
    # ---- training ----
    mlp = MLP(seed=args.seed)
    mlp.ymax = float(Tt.abs().max()) * 1.5   # clamp of the closure's outputs at run time
    zero = float((Tv ** 2).mean())
    _log({"samples": int(n), "data_s": out["data_s"], "val_loss_plain": zero})
    t1 = time.perf_counter()
    hist = train(mlp, Xt, Tt, epochs=args.epochs, batch=8192, lr=2e-3, val=(Xv, Tv), log=_log,
                 noise=args.noise, weight_decay=1e-4)
    torch.cuda.synchronize()
    out["train_s"] = time.perf_counter() - t1
    out["val_loss_plain"] = zero
    out["val_loss_closure"] = hist[-1]["val_loss"]
    out["train_history"] = hist
    # ---- held-out run: fine, plain coarse, coarse + closure to a common final time ----
    q = draws[-1]
    out["held_out"] = q
    fine, coarse = _problems(q, fine_res, coarse_res)
    out["fine_s"] = _timed(lambda: _run_to(fine, args.t_end))
    _, plain = _problems(q, fine_res, coarse_res)
    out["plain_s"] = _timed(lambda: _run_to(plain, args.t_end))
    # the one-step RHS error of plain coarse vs closure on the held-out draw's fine states
    Xh, Th = [], []
    _, ch = _problems(q, fine_res, coarse_res)
    fh, _ = _problems(q, fine_res, coarse_res)
    for _ in range(4):
        fh.stepper.run_steps(fh.f, fh.basis, fh.elliptic, fh.grids, fh.flux, fh.refs, args.every * 2)
        x, t = make_pair(fh, ch, proj, escale)
        Xh.append(x)
        Th.append(t)
    Xh, Th = torch.cat(Xh), torch.cat(Th)
    out["held_out_rhs_err_plain"] = float((Th ** 2).mean())
    out["held_out_rhs_err_closure"] = evaluate(mlp, Xh, Th)
    del fh, ch
    nsteps = plain.stepper.steps_counter
    _log({"fine_s": out["fine_s"], "plain_s": out["plain_s"], "coarse_steps": nsteps})
    ref = proj(fine.f.arr)
    tf, wf = np.asarray(fine.stepper.time_array), np.asarray(fine.stepper.field_energy)
    try:
        win = growth_window(tf, wf)
    except ValueError:
        win = (0.5 * args.t_end, args.t_end)
    g_f = growth_rate(tf, wf, *win)[0]

    def score(t, w, f):
        g = growth_rate(np.asarray(t), np.asarray(w), *win)[0]
        fi = f[1:-1, :, 1:-1, :, 1:-1, :].double()
        # compare at (about) the same final time: the coarse runs stop at their own last step
        l2 = float(torch.linalg.norm(fi - ref) / torch.linalg.norm(ref))
        return {"growth_rate": g, "growth_rate_rel_err": abs(g - g_f) / abs(g_f), "l2_rel_err": l2,
                "final_time": float(np.asarray(t)[-1])}

    out.update({"growth_window": list(win), "growth_rate_fine": g_f, "fine_final_time": float(tf[-1]),
                "fine_steps": int(fine.stepper.steps_counter), "coarse_steps": int(nsteps),
                "plain": score(plain.stepper.time_array, plain.stepper.field_energy, plain.f.arr)})
    runs = []
    for constraint in args.constraint:
        for alpha in args.alpha:
            _, cl = _problems(q, fine_res, coarse_res)
            cs = ClosureStepper(cl, mlp=mlp, escale=escale, alpha=alpha,
                                constraint=None if constraint == "none" else constraint)
            sec = _timed(lambda: cs.run_steps(nsteps, batch=50))
            rec = {"alpha": alpha, "constraint": constraint, "closure_s": sec, "fallback_step": cs.fallback_step,
                   "speedup_vs_fine": out["fine_s"] / sec, **score(cs.times, cs.energies, cl.f.arr)}
            _log(rec)
            runs.append(rec)
            del cs, cl
    out["closure_runs"] = runs
    # the first run under the earlier keys
    first = runs[0]
    out.update({"closure_s": first["closure_s"], "closure_fallback_step": first["fallback_step"],
                "closure": {k: first[k] for k in ("growth_rate", "growth_rate_rel_err", "l2_rel_err",
                                                  "final_time")},
                "speedup_closure_vs_fine": first["speedup_vs_fine"]})
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
