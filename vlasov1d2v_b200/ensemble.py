"""Batched heterogeneous ensembles: many independent Vlasov-Poisson runs in one set of launches.

``Ensemble(problems)`` takes problems built by ``problem.build`` (one precision; any grids,
orders 1..9 and physics) and advances all of them with the native ensemble driver
(``vl_ens_*`` in ``include/vlasov1d2v.h``): per RK stage one launch of each field-solve kernel
and one persistent stage kernel for every member together, K steps captured in one CUDA graph.
Each member keeps its own loop state, so members with different final times share a batch.

``autotune`` picks the ensemble's schedule -- threads per CTA, resident CTAs per SM and work
items per CTA -- by timing candidate schedules on the ensemble itself (states restored
afterwards), and caches the winner per ensemble signature and GPU in a JSON file.  A schedule
``(0, native, items_per_cta)`` is the by-order form (``vl_ens_schedule_by_order``): one stage
launch per order present, each kernel compiled for its order alone, except for the orders whose
bit n is set in ``native``, whose members run one by one through their own single-problem stage
kernel (the tensor-core kernel for n = 8, the generic kernel's TMA form on 16-byte rows);
``native = VL_ENS_NATIVE_AUTO`` selects the members whose kernels stage tiles by TMA.  The
launches of a stage run on concurrent streams.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os

import numpy as np
import torch

from . import _device, _lib
from .timestep import NonFiniteError, get_max_speeds

# by order, the members whose contexts stage tiles by TMA through their own single-problem
# kernels, 2 work items per CTA (the autotuner's choice on B200 for the 64-member benchmark)
DEFAULT_SCHEDULE = (0, _lib.VL_ENS_NATIVE_AUTO, 2)
_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "vlasov1d2v_b200", "ensemble_schedules.json")


class Ensemble:
    def __init__(self, problems, final_time=float("inf"), max_steps=2 ** 62, batch_steps=64):
        if not problems:
            raise ValueError("an ensemble needs at least one problem")
        self.problems = list(problems)
        self.batch = int(batch_steps)
        self.runs = []
        lib = _lib.load()
        finals = (list(final_time) if np.ndim(final_time) else [final_time] * len(self.problems))
        for p, fin in zip(self.problems, finals):
            st = p.stepper
            st.batch_steps = self.batch
            st.adapt_time_step(max_speeds=get_max_speeds(p.grids, p.elliptic, p.refs),
                               dx=p.grids.x.dx, du=p.grids.u.dx, dv=p.grids.v.dx)
            st.field_energy = np.append(st.field_energy, p.elliptic.electric_energy(grid=p.grids.x).get())
            run = st._run(p.f, p.elliptic, p.grids, p.refs)
            if run.background is not None:
                raise NotImplementedError("ensemble members run without the FP32 background split")
            run.upload_state(st._host_state(run, float(fin), max_steps))
            self.runs.append(run)
        handles = (ctypes.c_void_p * len(self.runs))(*[r.ctx.handle.value for r in self.runs])
        h = ctypes.c_void_p()
        _lib.check("vl_ens_create", lib.vl_ens_create(handles, len(self.runs), ctypes.byref(h)))
        self.handle = h
        self._lib = lib
        self.workspaces = []
        for i, r in enumerate(self.runs):
            nbytes = int(lib.vl_ens_workspace_bytes(h, i))
            ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=r.f.device)
            self.workspaces.append(ws)
            _lib.call("vl_ens_bind", h, i, r.f.data_ptr(), r.sa.data_ptr(), r.sb.data_ptr(),
                      r.E.data_ptr(), r.phi.data_ptr(), r.state.data_ptr(), ws.data_ptr())
        self.schedule = None
        self.set_schedule(*DEFAULT_SCHEDULE)
        self._graph = None
        self._graph_steps = 0

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._lib.vl_ens_destroy(h)
            except Exception:
                pass
            self.handle = None

    # -- schedule --------------------------------------------------------------------------------
    def set_schedule(self, threads, ctas_per_sm, items_per_cta):
        """threads 64 or 128 with ``ctas_per_sm`` resident CTAs: one stage kernel for all orders;
        threads 0: the by-order form, ``ctas_per_sm`` then the bit mask of the orders run through
        their members' own single-problem stage kernels."""
        if int(threads) == 0:
            _lib.call("vl_ens_schedule_by_order", self.handle, int(items_per_cta), int(ctas_per_sm))
        else:
            _lib.call("vl_ens_schedule", self.handle, int(threads), int(ctas_per_sm), int(items_per_cta))
        _lib.call("vl_ens_commit", self.handle)
        self.schedule = (int(threads), int(ctas_per_sm), int(items_per_cta))
        self._graph = None

    def signature(self):
        parts = [f"{r.ctx.nx}x{r.ctx.nu}x{r.ctx.nv}n{r.ctx.n}{r.ctx.precision}" for r in self.runs]
        name = torch.cuda.get_device_name(self.runs[0].f.device)
        return hashlib.sha1((name + "|" + ",".join(sorted(parts))).encode()).hexdigest()

    def _snapshot(self):
        return [(r.f.clone(), r.state.clone(), r.E.clone()) for r in self.runs]

    def _restore(self, snap):
        for r, (f, s, e) in zip(self.runs, snap):
            r.f.copy_(f)
            r.state.copy_(s)
            r.E.copy_(e)

    def time_schedule(self, schedule, steps=3, reps=2):
        """Device time (ms) per ensemble step of one schedule, best of ``reps``."""
        self.set_schedule(*schedule)
        stream = torch.cuda.current_stream()
        self._steps(1)   # warm-up (first launch of this configuration)
        best = float("inf")
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            self._steps(steps)
            b.record(stream)
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b) / steps)
        return best

    def autotune(self, candidates=None, steps=3, cache_path=_CACHE, use_cache=True):
        """Pick the fastest schedule for this ensemble; returns {"schedule", "ms", "trials"}.
        States, loop states and fields are restored after the trials."""
        key = self.signature()
        cache = {}
        if use_cache and cache_path and os.path.exists(cache_path):
            try:
                with open(cache_path) as fh:
                    cache = json.load(fh)
            except (OSError, ValueError):
                cache = {}
        if use_cache and key in cache:
            self.set_schedule(*cache[key]["schedule"])
            return cache[key]
        if candidates is None:
            candidates = [(t, c, k) for t in (128, 64) for c in (1, 2, 3, 4) for k in (1, 2, 4, 8)
                          if not (t == 128 and c > 2)]
            candidates += [(0, native, k) for native in (0, _lib.VL_ENS_NATIVE_AUTO) for k in (1, 2, 4, 8)]
            candidates += [(0, 0x3FE, 8)]   # every order through the single-problem kernels
        snap = self._snapshot()
        trials = []
        try:
            for cand in candidates:
                ms = self.time_schedule(cand, steps=steps)
                trials.append({"schedule": list(cand), "ms": ms})
                self._restore(snap)
        finally:
            self._restore(snap)
        best = min(trials, key=lambda r: r["ms"])
        self.set_schedule(*best["schedule"])
        out = {"schedule": best["schedule"], "ms": best["ms"], "trials": trials}
        if cache_path:
            try:
                os.makedirs(os.path.dirname(cache_path), exist_ok=True)
                cache[key] = out
                with open(cache_path, "w") as fh:
                    json.dump(cache, fh)
            except OSError:
                pass
        return out

    # -- stepping --------------------------------------------------------------------------------
    def _steps(self, nsteps):
        _lib.call("vl_ens_steps", self.handle, int(nsteps), ctypes.c_void_p(_device.stream_handle()))

    def launch(self, nsteps, use_graph=True):
        """Enqueue ``nsteps`` steps of every member (graph-replayed after the first capture)."""
        if not use_graph:
            self._steps(nsteps)
            return
        if self._graph is None or self._graph_steps != nsteps:
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    self._steps(nsteps)
            torch.cuda.current_stream().wait_stream(s)
            self._graph, self._graph_steps = g, nsteps
        self._graph.replay()

    def run_steps(self, nsteps, use_graph=True):
        """Advance every member by ``nsteps`` steps (fewer for members that reach their final
        time); each member's stepper receives its energy / time / dt histories."""
        remaining = int(nsteps)
        while remaining > 0:
            k = min(self.batch, remaining)
            for r, p in zip(self.runs, self.problems):
                st = r.read_state()
                st.steps = 0
                st.max_steps = k
                st.active_next = int(st.time < st.final_time and st.status == 0)
                r.upload_state(st)
            self.launch(k, use_graph)
            for r, p in zip(self.runs, self.problems):
                st = r.read_state()
                if st.status != 0:
                    raise NonFiniteError("non-finite field or energy in an ensemble member")
                h = r.hist[:, :int(st.steps)].cpu().numpy()
                stp = p.stepper
                for s in range(int(st.steps)):
                    stp.time = float(h[1, s])
                    stp.steps_counter += 1
                    stp.time_array = np.append(stp.time_array, stp.time)
                    stp.field_energy = np.append(stp.field_energy, h[0, s])
                    stp.dt = float(h[2, s])
            remaining -= k
        for r, p in zip(self.runs, self.problems):
            p.elliptic.electric_field = _device.wrap(r.E.clone())
            p.elliptic.potential = _device.wrap(r.phi.clone())

    def total_dof(self):
        return sum(r.ctx.nx * r.ctx.nu * r.ctx.nv * r.ctx.n ** 3 for r in self.runs)


def sample_members(count=64, seed=0, max_dof=2.4e6):
    """The seeded heterogeneous parameter set of the batched benchmark: k ~ U[0.5, 2] (gyroradius
    units), loss-cone index j in {3, 4, 5, 6}, omega_p / omega_c ~ U[5, 15], amplitude
    log-uniform in [1e-4, 1e-2], Nx in {8, 16, 32}, Nu = Nv in {24, 32, 40}, n in {6, 7, 8, 9},
    redrawn until the member has at most ``max_dof`` interior DOF."""
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        nx = int(rng.choice([8, 16, 32]))
        nuv = int(rng.choice([24, 32, 40]))
        n = int(rng.choice([6, 7, 8, 9]))
        k = float(rng.uniform(0.5, 2.0))
        j = int(rng.choice([3, 4, 5, 6]))
        ompc = float(rng.uniform(5.0, 15.0))
        amp = float(10 ** rng.uniform(-4.0, -2.0))
        if nx * nuv * nuv * n ** 3 > max_dof:
            continue
        out.append({"res": (nx, nuv, nuv), "order": n, "k": k, "ring_j": j, "om_pc": ompc, "amp": amp})
    return out


def build_members(params, precision="fp32", seed=0, batch_steps=64):
    from . import problem

    probs = []
    for i, q in enumerate(params):
        probs.append(problem.build(q["res"], q["order"], om_pc=q["om_pc"], k=q["k"], ring_j=q["ring_j"],
                                   perturbation="cos", amp=q["amp"], noise=0.0, seed=seed + i,
                                   precision=precision, batch_steps=batch_steps,
                                   background_split=False))
    return probs


__all__ = ["Ensemble", "sample_members", "build_members", "DEFAULT_SCHEDULE"]
