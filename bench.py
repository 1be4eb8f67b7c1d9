"""Benchmark: phase-space DOF-updates/s of the SSP-RK3 step (FP64 plain and FP32 mixed).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the medium benchmark configuration): Nx = 32, Nu = Nv = 50 elements, LGL order 8
(256 x 400 x 400 = 40.96M DOF), loss cone j = 6, perturbation 1e-3 cos kx plus seeded 1e-6
noise per x node, reference normalisation (omega_p / omega_c = 10, k = 0.886 gyroradius
units).  One step = one nonlinear SSP-RK3 step: 3 fused stage kernels + 3 field kernels.
Each state buffer (377 MB FP64 / 189 MB FP32) is larger than the 126 MB L2, so no flush is
needed between steps.  With N > 1 ranks (torchrun) every GPU advances its own replica (the
solver is single-GPU; replicas only): ``value`` is the sum over ranks, times are the max.

Variants in the same line: the FP32 mixed form of the same step, the large configuration
(64^3 elements, n = 9, 191M DOF; both precisions; single-GPU runs only) and the 64-member
heterogeneous FP32 ensemble.

Prints ONE JSON line (rank 0).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "phase-space DOF-updates/s per RK3 step, FP64 plain vs FP32 mixed; HBM roofline %"
RES = (32, 50, 50)
ORDER = 8
SAMPLE_RES = (4, 50, 50)  # labelled extra CPU sample: the same velocity grid, 4 of the 32 x elements


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="skip the batched-ensemble variant (64 heterogeneous FP32 members)")
    ap.add_argument("--ensemble-steps", type=int, default=50)
    ap.add_argument("--ensemble-only", action="store_true",
                    help="measure the batched-ensemble variant alone (profiling target)")
    ap.add_argument("--ensemble-schedule", type=int, nargs=3, default=None,
                    metavar=("THREADS", "CTAS_PER_SM", "ITEMS_PER_CTA"),
                    help="fixed ensemble schedule instead of the autotuner (threads 0: by order)")
    ap.add_argument("--no-large", action="store_true",
                    help="skip the large-configuration variant (64^3 elements, n = 9)")
    ap.add_argument("--kernel-reps", type=int, default=10)
    ap.add_argument("--kernel-only", action="store_true",
                    help="launch each stage kind --kernel-reps times on --res (profiling target)")
    ap.add_argument("--res", type=int, nargs=3, default=list(RES))
    ap.add_argument("--order", type=int, default=ORDER)
    ap.add_argument("--precision", choices=("fp64", "fp32"), default="fp64")
    return ap.parse_args()


def kernel_only(args):
    """Plain launches of the three fused stage kinds, the standalone moment and one field solve
    per repetition (no graphs, no timing of its own): the target of ncu captures of single
    kernels."""
    import torch

    from vlasov1d2v_b200 import problem
    from vlasov1d2v_b200.context import get_context

    torch.cuda.set_device(0)
    res, n = tuple(args.res), args.order
    p = problem.build(res, n, perturbation="cos", amp=1.0e-3, noise=1.0e-6, seed=0,
                      precision=args.precision)
    ctx = get_context(p.grids, precision=args.precision, accel=p.refs.electron_acceleration_multiplier,
                      bfield=p.elliptic.magnetic_field, kappa=p.elliptic.poisson_coefficient,
                      courant=p.stepper.courant)
    f = p.f.arr.as_subclass(torch.Tensor)
    sa, sb = torch.empty_like(f), torch.empty_like(f)
    ctx.sync_ghosts(f, sa)
    ctx.sync_ghosts(f, sb)
    E = p.elliptic.electric_field.as_subclass(torch.Tensor).contiguous()
    dt = torch.tensor([1.0e-3], dtype=torch.float64, device=f.device)
    if getattr(p.f, "background_split", False) and p.f.background is not None:
        # the FP32 mixed form's stage kernels also read the background RHS tables
        ctx.set_background(p.f.background_tables(p.grids, p.refs.electron_acceleration_multiplier,
                                                 p.elliptic.magnetic_field))
    rho = torch.zeros((res[0], n), dtype=torch.float64, device=f.device)
    phi = torch.empty_like(rho)
    for _ in range(args.kernel_reps):
        ctx.rk_stage(0, f, None, sa, E, dt, partials=ctx.workspace)
        ctx.rk_stage(1, sa, f, sb, E, dt, partials=ctx.workspace)
        ctx.rk_stage(2, sb, f, sa, E, dt, partials=ctx.workspace)
        # the standalone moment and the cluster field solve of the same problem
        ctx.moment(f, rho)
        ctx.poisson((rho.mean() - rho).contiguous(), E, phi)
    torch.cuda.synchronize()
    print(json.dumps({"kernel_only": True, "res": list(res), "order": n, "precision": args.precision,
                      "reps": args.kernel_reps,
                      "background_split": bool(getattr(p.f, "background_split", False)),
                      "state_mb": f.numel() * f.element_size() / 1e6}))
    return 0


def dof(res, n):
    return res[0] * res[1] * res[2] * n ** 3


# ----------------------------------------------------------------------------------------------
# CPU (oracle port) timing: the reference arm and the cpu_baseline object
# ----------------------------------------------------------------------------------------------
def cpu_port_rate(steps, warmup, res=RES):
    """Steps of the oracle port (NumPy FP64 restatement of the reference step, BLAS on every host
    core) on the benchmark grid itself: DOF-updates/s, seconds per step, cores."""
    import numpy as np

    from oracle import vlasov_oracle as vo

    c = vo.make_case(*res, ORDER)
    f = vo.cos_perturbed(c, c.extra["norm"].vt_e, 6, 1.0e-3, noise=1.0e-6, seed=0)
    rho = vo.moment_zero(f, c)
    E0, _ = vo.poisson2(rho - np.mean(rho), c)
    dt = vo.adapt_dt(E0, c)
    for _ in range(warmup):
        _, dt = vo.ssp_rk3_step(f, dt, c)
    t0 = time.perf_counter()
    for _ in range(steps):
        _, dt = vo.ssp_rk3_step(f, dt, c)
    t = (time.perf_counter() - t0) / max(steps, 1)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    return dof(res, ORDER) / t, t, cores


def measure_ensemble(steps, warmup, members=64, seed=0, schedule=None):
    """Batched heterogeneous ensemble (64 seeded FP32 members, orders 6-9, up to 2.4M DOF each):
    aggregate DOF-updates/s of the ensemble driver (schedule from the autotuner), and of the same
    members stepped one after another through the single-problem loop (each graph-captured)."""
    import torch

    from vlasov1d2v_b200.ensemble import Ensemble, build_members, sample_members

    params = sample_members(members, seed=seed)
    t0 = time.perf_counter()
    probs = build_members(params, precision="fp32", seed=seed, batch_steps=max(steps, warmup))
    ens = Ensemble(probs, batch_steps=max(steps, warmup))
    setup_s = time.perf_counter() - t0
    if schedule is None:
        tune = ens.autotune(steps=3, use_cache=False, cache_path=None)
    else:
        ens.set_schedule(*schedule)
        tune = {"schedule": list(schedule), "trials": []}
    total = ens.total_dof()
    ens.launch(warmup, use_graph=False)
    ens.launch(steps, use_graph=True)   # capture
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    ens.launch(steps, use_graph=True)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    # the same members one after another, each through its own graph-captured loop
    seq_ms = 0.0
    for r in ens.runs:
        r.launch(warmup, use_graph=False)
        r.launch(steps, use_graph=True)
        torch.cuda.synchronize()
        c, d = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c.record()
        r.launch(steps, use_graph=True)
        d.record()
        torch.cuda.synchronize()
        seq_ms += c.elapsed_time(d) / steps
        r.graph = None
    orders = sorted({r.ctx.n for r in ens.runs})
    return {"value": total / (ms * 1e-3), "unit": "DOF-updates/s", "dtype": "f32",
            "ms_per_step": ms, "members": len(ens.runs), "total_dof": total, "orders": orders,
            "schedule": tune["schedule"], "autotune_trials": len(tune["trials"]),
            "sequential_single_runs_value": total / (seq_ms * 1e-3),
            "speedup_vs_sequential": seq_ms / ms, "setup_s": setup_s,
            "workload": "64 seeded loss-cone members: k~U[0.5,2], j in {3..6}, wp/wc~U[5,15], "
                        "amp log-U[1e-4,1e-2], Nx in {8,16,32}, Nu=Nv in {24,32,40}, n in {6..9}, "
                        "<= 2.4M DOF each"}


def cpu_baseline_obj(steps=2, warmup=1):
    """The CPU path timed on the benchmark configuration itself (same grid, same initial state),
    plus the x-slab sample of earlier runs as a labelled extra."""
    rate, t, cores = cpu_port_rate(steps, warmup)
    srate, st, _ = cpu_port_rate(3, 1, res=SAMPLE_RES)
    return {"value": rate, "unit": "DOF-updates/s", "cores": cores, "kind": "port", "same_config": True,
            "sample": f"oracle (NumPy FP64 restatement of the reference step) on the full benchmark grid "
                      f"Nx={RES[0]}, Nu=Nv={RES[1]}, n={ORDER} ({dof(RES, ORDER)/1e6:.2f}M DOF), "
                      f"{steps} steps after {warmup} warm-up, {t:.2f} s/step; BLAS threads = cores, "
                      "elementwise NumPy single-threaded",
            "slab_sample": {"value": srate, "res": list(SAMPLE_RES), "s_per_step": st}}


# ----------------------------------------------------------------------------------------------
# clocks sampling (nvidia-smi during the timed region)
# ----------------------------------------------------------------------------------------------
class Clocks:
    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"vl_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "samples": len(sm),
                "reasons": sorted(reasons)}


# ----------------------------------------------------------------------------------------------
# GPU measurement
# ----------------------------------------------------------------------------------------------
STAGE_PROFILES = {"fp64": "stage_frag_fp64_16x50x50_n8.md", "fp32": "stage_f32_fp32_16x50x50_n8.md"}


def profiled_traffic_ratio(precision):
    """DRAM bytes (read + write) per algorithmic byte of one fused stage launch, from the ncu
    capture summarised in profiles/ for the benchmark's stage kernel of that precision (a
    half-size case of the same kernel; the traffic scales with the elements processed).  None
    when absent."""
    import re
    path = os.path.join(ROOT, "profiles", STAGE_PROFILES[precision])
    try:
        text = open(path).read()
    except OSError:
        return None, None
    m = re.search(r"DRAM read / write \| ([0-9.]+) / ([0-9.]+) MB", text)
    a = re.search(r"write s_\(i\+1\) = \d+ B/DOF = ([0-9.]+) MB", text)
    if not m or not a:
        return None, None
    return (float(m.group(1)) + float(m.group(2))) / float(a.group(1)), os.path.relpath(path, ROOT)


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s (of fallback)"


def capture_steps(run, steps):
    """CUDA graph of `steps` SSP-RK3 steps of a Stepper run.  The FP32 mixed form's
    background-split tables are installed on the context while the graph is captured, so the
    captured stage kernels carry them, as in Stepper launches."""
    import torch

    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    run.ctx.set_background(run.background)
    try:
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                run.ctx.ssp_rk3_steps(run.f, run.sa, run.sb, run.E, run.phi, run.state, steps)
    finally:
        run.ctx.set_background(None)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    return g


def measure_precision(precision, steps, warmup, reps, dist, res=None, order=None, e2e=True):
    import torch

    from vlasov1d2v_b200 import problem
    from vlasov1d2v_b200.timestep import _BIG_STEPS, get_max_speeds

    res = tuple(res or RES)
    order = order or ORDER
    p = problem.build(res, order, perturbation="cos", amp=1.0e-3, noise=1.0e-6, seed=0,
                      precision=precision, batch_steps=max(steps, warmup, 1))
    st = p.stepper
    st.adapt_time_step(max_speeds=get_max_speeds(p.grids, p.elliptic, p.refs),
                       dx=p.grids.x.dx, du=p.grids.u.dx, dv=p.grids.v.dx)
    run = st._run(p.f, p.elliptic, p.grids, p.refs)
    run.upload_state(st._host_state(run, float("inf"), _BIG_STEPS))
    n_dof = dof(res, order)
    es = 8 if precision == "fp64" else 4

    # warm-up (eager), then capture the K-step graph
    if warmup:
        run.launch(warmup, use_graph=False)
    torch.cuda.synchronize()
    g = capture_steps(run, steps)

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    ev0.record()
    g.replay()
    ev1.record()
    torch.cuda.synchronize()
    dist.barrier()
    ms = ev0.elapsed_time(ev1)
    stt = run.read_state()
    if stt.status != 0:
        raise RuntimeError("non-finite state during the benchmark")

    # per-kernel timing of the three stage kinds (the dominant kernel) with CUDA events, the
    # same kernel instantiations as the loop's (FP32: with the background-split tables)
    ctx = run.ctx
    dt_t = torch.tensor([float(stt.dt)], dtype=torch.float64, device=run.f.device)
    stage_ms = []
    ctx.set_background(run.background)
    try:
        for stage, inp, fn, out in ((0, run.f, None, run.sa), (1, run.sa, run.f, run.sb),
                                    (2, run.sb, run.f, run.sa)):
            for _ in range(2):
                ctx.rk_stage(stage, inp, fn, out, run.E, dt_t, partials=ctx.workspace)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                ctx.rk_stage(stage, inp, fn, out, run.E, dt_t, partials=ctx.workspace)
            b.record()
            torch.cuda.synchronize()
            stage_ms.append(a.elapsed_time(b) / reps)
    finally:
        ctx.set_background(None)
    # field solve (one 8-CTA cluster: Poisson solve from a density)
    rho = torch.zeros((res[0], order), dtype=torch.float64, device=run.f.device)
    ctx.moment(run.f, rho)
    chg = (rho.mean() - rho).contiguous()
    phi = torch.empty_like(rho)
    for _ in range(2):
        ctx.poisson(chg, run.E, phi)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        ctx.poisson(chg, run.E, phi)
    b.record()
    torch.cuda.synchronize()
    field_ms = a.elapsed_time(b) / reps

    state_bytes = run.f.numel() * es
    if not e2e:
        del g
        return {"precision": precision, "ms": ms, "steps": steps, "dof": n_dof, "bytes_per_dof_step": 8 * es,
                "stage_ms": stage_ms, "field_ms": field_ms, "state_bytes": state_bytes,
                "stage_bytes": [2 * es * n_dof, 3 * es * n_dof, 3 * es * n_dof]}
    # end to end through the public API with host buffers: pinned f0 -> device, K steps,
    # device -> host of the final state and of the per-step energy/time/dt histories
    host_f = torch.empty(run.f.shape, dtype=run.f.dtype, pin_memory=True)
    host_f.copy_(run.f)
    host_h = torch.empty((3, steps), dtype=torch.float64, pin_memory=True)
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run.f.copy_(host_f, non_blocking=True)
    g.replay()
    host_f.copy_(run.f, non_blocking=True)
    host_h.copy_(run.hist[:, :steps], non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    dist.barrier()
    e2e_ms = e0.elapsed_time(e1)
    state_bytes = run.f.numel() * es
    del g
    return {
        "precision": precision, "ms": ms, "steps": steps, "dof": n_dof, "bytes_per_dof_step": 8 * es,
        "stage_ms": stage_ms, "field_ms": field_ms, "e2e_ms": e2e_ms, "state_bytes": state_bytes,
        "stage_bytes": [2 * es * n_dof, 3 * es * n_dof, 3 * es * n_dof],
    }


LARGE_RES, LARGE_ORDER = (64, 64, 64), 9


def measure_large(steps, warmup, dist, peak):
    """The large benchmark configuration (64^3 elements, n = 9, 191M DOF; FP64 plain and FP32
    mixed): DOF-updates/s of the graph-replayed step and each stage kernel's fraction of the HBM
    roofline (the FP64 stage kernel is the generic kernel's TMA form, the FP32 one the
    register-pencil kernel)."""
    out = {"workload": "large loss-cone config: Nx=Nu=Nv=64, n=9 (576^3 = 191.1M DOF), "
                       "1e-3 cos kx + 1e-6 noise"}
    for prec in ("fp64", "fp32"):
        r = measure_precision(prec, steps, warmup, 3, dist, res=LARGE_RES, order=LARGE_ORDER, e2e=False)
        ms_step = r["ms"] / steps
        fr = [b / (t * 1e-3) / (peak * 1e9) for b, t in zip(r["stage_bytes"], r["stage_ms"])]
        out[prec] = {"value": r["dof"] / (ms_step * 1e-3), "unit": "DOF-updates/s", "ms_per_step": ms_step,
                     "stage_ms": r["stage_ms"], "stage_roofline_frac": fr,
                     "step_roofline_frac": r["bytes_per_dof_step"] * r["dof"] / (ms_step * 1e-3) / (peak * 1e9)}
    return out


def replica_throughput(dist, ms, steps, dof):
    """Whole-job throughput of independent replicas: the step time is the slowest rank's
    (max over ranks of the device-timed region), the value the sum of every rank's DOF over it."""
    ms_step = dist.max(ms) / steps
    return ms_step, dist.sum(dof / (ms_step * 1e-3))


class _NoDist:
    def barrier(self):
        pass

    def max(self, x):
        return x

    def sum(self, x):
        return x


class _TorchDist:
    def __init__(self, torch, dist, device="cuda"):
        self.t = torch
        self.d = dist
        self.device = device

    def barrier(self):
        self.d.barrier()

    def _reduce(self, x, op):
        v = self.t.tensor([float(x)], dtype=self.t.float64, device=self.device)
        self.d.all_reduce(v, op=op)
        return float(v.item())

    def max(self, x):
        return self._reduce(x, self.d.ReduceOp.MAX)

    def sum(self, x):
        return self._reduce(x, self.d.ReduceOp.SUM)


def main():
    args = parse()
    if args.kernel_only:
        return kernel_only(args)
    if args.ensemble_only:
        import torch

        torch.cuda.set_device(0)
        res = measure_ensemble(args.ensemble_steps, args.warmup, schedule=args.ensemble_schedule)
        print(json.dumps({"ensemble_only": True, "ensemble_fp32": res}))
        return 0
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        # the reference's CPU path (oracle port, all host threads) on rank 0 only, on the benchmark
        # grid itself: at most 3 timed steps after at most 1 warm-up step (about 13-17 s per step on
        # 8 host cores), whatever K and W are, so the arm ends within a few minutes
        if rank != 0:
            return 0
        ksteps, kwarm = max(1, min(args.steps, 3)), min(args.warmup, 1)
        rate, t, cores = cpu_port_rate(ksteps, kwarm)
        sample = (f"oracle (NumPy FP64 restatement of the reference step) on the full benchmark grid "
                  f"Nx={RES[0]}, Nu=Nv={RES[1]}, n={ORDER}; {ksteps} timed steps after {kwarm} warm-up, "
                  f"{t:.2f} s/step")
        line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "DOF-updates/s",
                "n_gpus": args.gpus, "steps": ksteps, "warmup": kwarm,
                "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "medium loss-cone config: Nx=32, Nu=Nv=50, LGL n=8 "
                                       "(256x400x400 = 40.96M DOF), j=6, 1e-3 cos kx + 1e-6 noise",
                           "dof": dof(RES, ORDER), "same_config": True},
                "cpu_baseline": {"value": rate, "unit": "DOF-updates/s", "cores": cores,
                                 "kind": "port", "sample": sample},
                "e2e": {"value": rate, "unit": "DOF-updates/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch

    if world > 1:
        import torch.distributed as tdist
        from datetime import timedelta

        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = _TorchDist(torch, tdist)
    else:
        torch.cuda.set_device(0)
        dist = _NoDist()

    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    phys = int(vis.split(",")[local]) if vis and vis.split(",")[local].strip().isdigit() else local
    results = {}
    clocks = Clocks(phys)
    with clocks:
        for prec in ("fp64", "fp32"):
            results[prec] = measure_precision(prec, args.steps, args.warmup, args.kernel_reps, dist)
            torch.cuda.empty_cache()
    ck = clocks.summary()

    peak, peak_src = measured_peak_hbm()
    out = {}
    for prec, r in results.items():
        ms_step, value = replica_throughput(dist, r["ms"], r["steps"], r["dof"])
        stage_s = sum(r["stage_ms"]) * 1e-3
        achieved = sum(r["stage_bytes"]) / stage_s / 1e9
        ratio, tsrc = profiled_traffic_ratio(prec)
        per_launch = sum(r["stage_bytes"]) / len(r["stage_bytes"])
        e2e_s = dist.max(r["e2e_ms"]) * 1e-3
        out[prec] = {
            "value": value, "ms_per_step": ms_step,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": None if ratio is None else ratio * per_launch,
                         "traffic_note": None if ratio is None else
                         f"bytes per launch (mean of the 3 stage kinds) = algorithmic x {ratio:.3f}, "
                         f"the DRAM/algorithmic ratio of the ncu capture in {tsrc}",
                         "algorithmic_bytes_per_launch": per_launch,
                         "kernel": "stage_frag_kernel<double>" if prec == "fp64" else
                                   "stage_f32_kernel<kind, background split>",
                         "algorithmic_bytes_per_dof_step": r["bytes_per_dof_step"],
                         "stage_ms": r["stage_ms"], "field_ms": r["field_ms"],
                         "step_effective_gbs": r["dof"] * r["bytes_per_dof_step"] / (ms_step * 1e-3) / 1e9,
                         "peak_source": peak_src},
            "e2e": {"value": dist.sum(r["dof"] * r["steps"] / e2e_s), "unit": "DOF-updates/s",
                    "h2d_bytes_per_step": r["state_bytes"] / r["steps"],
                    "d2h_bytes_per_step": (r["state_bytes"] + 24 * r["steps"]) / r["steps"],
                    "copies": f"the state copied host->device once and device->host once per "
                              f"K={r['steps']} steps (a time loop's input and result), plus each "
                              "step's energy, time and dt; bytes per step = job bytes / K"},
        }
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0
    head = out["fp64"]
    line = {
        "metric": METRIC, "value": head["value"], "unit": "DOF-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "medium loss-cone config: Nx=32, Nu=Nv=50, LGL n=8 "
                               "(256x400x400 = 40.96M DOF per GPU), j=6, 1e-3 cos kx + 1e-6 noise, "
                               "nonlinear SSP-RK3 + spectral Poisson per stage",
                   "dof_per_gpu": dof(RES, ORDER), "l2": "inputs larger than L2 (377 MB FP64 state "
                   "buffers, 3 buffers)", "parallelism": f"replicas x{world}"},
        "roofline": head["roofline"],
        "e2e": head["e2e"],
        # per step: 3 fused stage kernels + 3 cluster field solves; one moment per call
        "gpu_launches": 6 * args.steps + 1,
        "clocks": ck,
        "variants": {"fp32_mixed": {"value": out["fp32"]["value"], "dtype": "f32",
                                    "ms_per_step": out["fp32"]["ms_per_step"],
                                    "roofline": out["fp32"]["roofline"], "e2e": out["fp32"]["e2e"],
                                    "speedup_vs_fp64": out["fp32"]["value"] / head["value"]}},
    }
    if not args.no_large and world == 1:
        try:
            line["variants"]["large_n9"] = measure_large(min(args.steps, 10), args.warmup, dist, peak)
        except Exception as exc:   # the headline line is still printed
            line["variants"]["large_n9"] = {"error": f"{type(exc).__name__}: {exc}"}
    if not args.no_ensemble:
        try:
            line["variants"]["ensemble_fp32"] = measure_ensemble(args.ensemble_steps, args.warmup,
                                                                 schedule=args.ensemble_schedule)
        except Exception as exc:  # the headline line must survive a failure of the extra
            line["variants"]["ensemble_fp32"] = {"error": f"{type(exc).__name__}: {exc}"}
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline_obj()
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
