"""SSP-RK3 time stepping of the 1D2V Vlasov-Poisson system.

Mirrors ``Stepper`` and ``get_max_speeds`` of crewsdw/Vlasov1D2V (``main/timestep.py``).

``main_loop`` runs the nonlinear SSP-RK3 loop (``main/timestep.py:81-187``) on the device: per
step three fused stage kernels (RHS + RK combination + moment partials of the result) and
three field solves, each one 8-CTA thread-block cluster (density -> Poisson -> E, plus energy,
dt and the loop bookkeeping after stage 2).  The loop state (dt, time, step count, "keep going" flag, energy
and time histories) lives in device memory, so batches of steps run without host syncs and,
after the first batch, as a replayed CUDA graph.  The host reads the histories back once per
batch and fills ``time_array`` / ``field_energy`` exactly as the reference's loop does,
including its quirks: the energy recorded after a step is that of the field of RK stage s1,
and ``time`` advances by the dt adapted at the end of the step.
"""
from __future__ import annotations

import ctypes
import time as timer

import numpy as np
import torch

from . import _device, _lib
from .context import get_context

ssp_rk_switch = {
    1: [1],
    2: [1 / 2, 1 / 2],
    3: [1 / 3, 1 / 2, 1 / 6],
    4: [3 / 8, 1 / 3, 1 / 4, 1 / 24],
    5: [11 / 30, 3 / 8, 1 / 6, 1 / 12, 1 / 120],
    6: [53 / 144, 11 / 30, 3 / 16, 1 / 18, 1 / 48, 1 / 720],
    7: [103 / 280, 53 / 144, 11 / 60, 3 / 48, 1 / 72, 1 / 240, 1 / 5040],
    8: [2119 / 5760, 103 / 280, 53 / 288, 11 / 180, 1 / 64, 1 / 360, 1 / 1440, 1 / 40320],
}

# Cockburn & Shu (2001) RK-DG Courant numbers, [time_order][space_order - 1]
courant_numbers = {
    1: [1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0],
    2: [1.0, 0.333],
    3: [1.256, 0.409, 0.209, 0.130, 0.089, 0.066, 0.051, 0.040, 0.033],
    4: [1.392, 0.464, 0.235, 0.145, 0.100, 0.073, 0.056, 0.045, 0.037],
    5: [1.608, 0.534, 0.271, 0.167, 0.115, 0.085, 0.065, 0.052, 0.042],
    6: [1.776, 0.592, 0.300, 0.185, 0.127, 0.093, 0.072, 0.057, 0.047],
    7: [1.977, 0.659, 0.333, 0.206, 0.142, 0.104, 0.080, 0.064, 0.052],
    8: [2.156, 0.718, 0.364, 0.225, 0.154, 0.114, 0.087, 0.070, 0.057],
}

nonlinear_ssp_rk_switch = {
    2: [[1 / 2, 1 / 2, 1 / 2]],
    3: [[3 / 4, 1 / 4, 1 / 4], [1 / 3, 2 / 3, 2 / 3]],
}

_BIG_STEPS = 2 ** 62


class NonFiniteError(FloatingPointError):
    """The device loop detected a non-finite density, field, energy or dt."""


class _Run:
    """Device buffers of one (distribution, grids, physics) loop set-up."""

    def __init__(self, ctx, f, hist_cap):
        dev = f.device
        self.ctx = ctx
        self.f = f
        self.sa = torch.empty_like(f)
        self.sb = torch.empty_like(f)
        self.E = torch.zeros((ctx.nx + 2, ctx.n), dtype=torch.float64, device=dev)
        self.phi = torch.zeros((ctx.nx, ctx.n), dtype=torch.float64, device=dev)
        self.state = torch.zeros(_lib.RUN_STATE_BYTES, dtype=torch.uint8, device=dev)
        self.hist = torch.zeros((3, hist_cap), dtype=torch.float64, device=dev)
        self.cap = hist_cap
        self.graph = None
        self.graph_steps = 0
        self.synced_ptr = None
        self.background = None   # RHS tables of the FP32 background split, or None

    def upload_state(self, st: _lib.VlRunState):
        host = torch.frombuffer(bytearray(bytes(st)), dtype=torch.uint8)
        self.state.copy_(host, non_blocking=False)

    def read_state(self) -> _lib.VlRunState:
        raw = self.state.cpu().numpy().tobytes()
        return _lib.VlRunState.from_buffer_copy(raw)

    def sync_ghosts(self):
        self.ctx.sync_ghosts(self.f, self.sa)
        self.ctx.sync_ghosts(self.f, self.sb)
        self.synced_ptr = self.f.data_ptr()

    def launch(self, nsteps, use_graph):
        # the background tables ride in the stage kernels' launch parameters: install them on
        # the (shared) context for these launches only
        self.ctx.set_background(self.background)
        try:
            self._launch(nsteps, use_graph)
        finally:
            self.ctx.set_background(None)

    def _launch(self, nsteps, use_graph):
        if not use_graph:
            self.ctx.ssp_rk3_steps(self.f, self.sa, self.sb, self.E, self.phi, self.state, nsteps)
            return
        if self.graph is None or self.graph_steps != nsteps:
            # warm the launch path once outside capture, then capture nsteps steps
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    self.ctx.ssp_rk3_steps(self.f, self.sa, self.sb, self.E, self.phi, self.state,
                                           nsteps)
            torch.cuda.current_stream().wait_stream(s)
            self.graph = g
            self.graph_steps = nsteps
        self.graph.replay()


class Stepper:
    def __init__(self, time_order, space_order, write_time, final_time, linear=False,
                 batch_steps=32, use_graph=True, verbose=True):
        self.time_order = time_order
        self.space_order = space_order
        self.linear = linear
        if linear:
            self.coefficients = self.get_coefficients()
        else:
            self.coefficients = self.get_nonlinear_coefficients()
        self.courant = self.get_courant_number()
        self.time = 0
        self.dt = None
        self.steps_counter = 0
        self.write_counter = 1
        self.write_time = write_time
        self.final_time = final_time
        self.time_array = np.array([self.time])
        self.field_energy = np.array([])
        self.batch_steps = int(batch_steps)
        self.use_graph = bool(use_graph)
        self.verbose = bool(verbose)
        self._runs = {}

    def get_coefficients(self):
        return np.array([ssp_rk_switch.get(self.time_order, "nothing")][0])

    def get_nonlinear_coefficients(self):
        return np.array(nonlinear_ssp_rk_switch.get(self.time_order, "nothing"))

    def get_courant_number(self):
        return courant_numbers.get(self.time_order)[self.space_order - 1]

    # ------------------------------------------------------------------------------------------
    def _context(self, distribution, elliptic, grids, refs):
        f = _device.plain(distribution.arr)
        return get_context(grids, precision=_device.precision_of(f),
                           accel=refs.electron_acceleration_multiplier,
                           bfield=elliptic.magnetic_field, kappa=elliptic.poisson_coefficient,
                           courant=self.courant)

    def _run(self, distribution, elliptic, grids, refs):
        if self.time_order != 3 or self.linear:
            raise NotImplementedError("the native loop implements the nonlinear SSP-RK3 stepper")
        ctx = self._context(distribution, elliptic, grids, refs)
        f = _device.plain(distribution.arr)
        if not f.is_contiguous():
            distribution.arr = _device.wrap(f.contiguous())
            f = _device.plain(distribution.arr)
        key = (id(ctx), f.data_ptr())
        run = self._runs.get(key)
        if run is None:
            run = _Run(ctx, f, hist_cap=max(self.batch_steps, 1))
            self._runs = {key: run}
        if getattr(distribution, "background_split", False) and distribution.background is not None:
            run.background = distribution.background_tables(
                grids, refs.electron_acceleration_multiplier, elliptic.magnetic_field)
        else:
            run.background = None
        # stage buffers take f's ghost elements (the inflow boundary values) and f gets the
        # periodic x-ghost swap, as main/timestep.py:143-151 does at every step
        run.sync_ghosts()
        return run

    def _host_state(self, run, final_time, max_steps):
        st = _lib.VlRunState()
        st.dt = float(self.dt)
        st.dt_next = float(self.dt)
        st.time = float(self.time)
        st.final_time = float(final_time)
        st.steps = 0
        st.max_steps = int(max_steps)
        st.active = 0
        st.active_next = int((st.time < st.final_time) and (st.max_steps > 0))
        st.status = 0
        st.hist_capacity = run.cap
        st.energy_hist = run.hist[0].data_ptr()
        st.time_hist = run.hist[1].data_ptr()
        st.dt_hist = run.hist[2].data_ptr()
        return st

    def resume_from(self, checkpoint, distribution, elliptic):
        """Restore a checkpoint written by ``RunData.save_checkpoint`` (a dict as returned by
        ``ReadData.read_checkpoint``): the state, the field and potential, the clock, dt, the
        counters and the histories.  The next ``main_loop`` / ``run_steps`` continues the saved
        run exactly (no initial energy entry, no dt re-adaptation)."""
        distribution.set_array(checkpoint["f"])
        elliptic.electric_field = _device.wrap(_device.as_tensor(checkpoint["E"]).clone())
        elliptic.potential = _device.wrap(_device.as_tensor(checkpoint["phi"]).clone())
        self.time = float(checkpoint["time"])
        self.dt = float(checkpoint["dt"])
        self.steps_counter = int(checkpoint["steps"])
        self.write_counter = int(checkpoint["write_counter"])
        self.time_array = np.array(checkpoint["time_array"], dtype=np.float64)
        self.field_energy = np.array(checkpoint["field_energy"], dtype=np.float64)
        self._resumed = True

    def main_loop(self, distribution, basis, elliptic, grids, dg_flux, refs, save_file):
        t0 = timer.time()
        if getattr(self, "_resumed", False):
            self._resumed = False
        else:
            self.field_energy = np.append(self.field_energy, elliptic.electric_energy(grid=grids.x).get())
            if self.verbose:
                print('\nInitializing time-step...')
            self.adapt_time_step(max_speeds=get_max_speeds(grids, elliptic, refs),
                                 dx=grids.x.dx, du=grids.u.dx, dv=grids.v.dx)
        run = self._run(distribution, elliptic, grids, refs)
        run.upload_state(self._host_state(run, self.final_time, _BIG_STEPS))
        batches = 0
        while True:
            k = self.batch_steps
            run.launch(k, self.use_graph and batches > 0)
            batches += 1
            st = run.read_state()
            new = int(st.steps)
            if new > 0:
                h = run.hist[:, :new].cpu().numpy() if new <= run.cap else None
                if h is None:
                    raise RuntimeError("history ring overflow")
                for s in range(new):
                    self.time = float(h[1, s])
                    self.steps_counter += 1
                    self.time_array = np.append(self.time_array, self.time)
                    self.field_energy = np.append(self.field_energy, h[0, s])
                    self.dt = float(h[2, s])
                    if self.time > self.write_counter * self.write_time:
                        self.write_counter += 1
                        if self.verbose:
                            print('\nI made it through step ' + str(self.steps_counter))
                            print('The simulation time is {:0.3e}'.format(self.time))
                            print('The time-step is {:0.3e}'.format(self.dt))
                            print('Time since start is ' + str((timer.time() - t0) / 60.0) + ' minutes')
            if st.status != 0:
                raise NonFiniteError(
                    f"non-finite field or energy detected by step {self.steps_counter}")
            if not st.active_next:
                break
            # the history ring holds one batch: rebase the device step counter
            st2 = _lib.VlRunState.from_buffer_copy(bytes(st))
            st2.steps = 0
            st2.max_steps = _BIG_STEPS
            run.upload_state(st2)
        elliptic.electric_field = _device.wrap(run.E.clone())
        elliptic.potential = _device.wrap(run.phi.clone())
        if self.verbose:
            print('\nFinal time reached')
            print('Total steps were ' + str(self.steps_counter))
            print('Time since start is {:0.3e}'.format(timer.time() - t0))

    def run_steps(self, distribution, basis, elliptic, grids, dg_flux, refs, nsteps):
        """Advance exactly ``nsteps`` steps (no final-time test) with the main loop's
        bookkeeping: energies and times appended, initial energy/dt from the current field."""
        if getattr(self, "_resumed", False):
            self._resumed = False
        elif self.dt is None or len(self.field_energy) == 0:
            self.field_energy = np.append(self.field_energy,
                                          elliptic.electric_energy(grid=grids.x).get())
            self.adapt_time_step(max_speeds=get_max_speeds(grids, elliptic, refs),
                                 dx=grids.x.dx, du=grids.u.dx, dv=grids.v.dx)
        saved_final, saved_verbose = self.final_time, self.verbose
        remaining = int(nsteps)
        run = self._run(distribution, elliptic, grids, refs)
        while remaining > 0:
            k = min(self.batch_steps, remaining)
            run.upload_state(self._host_state(run, float("inf"), k))
            run.launch(k, False)
            st = run.read_state()
            h = run.hist[:, :int(st.steps)].cpu().numpy()
            for s in range(int(st.steps)):
                self.time = float(h[1, s])
                self.steps_counter += 1
                self.time_array = np.append(self.time_array, self.time)
                self.field_energy = np.append(self.field_energy, h[0, s])
                self.dt = float(h[2, s])
            if st.status != 0:
                raise NonFiniteError("non-finite field or energy detected")
            remaining -= int(st.steps)
        self.final_time, self.verbose = saved_final, saved_verbose
        elliptic.electric_field = _device.wrap(run.E.clone())
        elliptic.potential = _device.wrap(run.phi.clone())

    def nonlinear_ssp_rk(self, distribution, basis, elliptic, grids, dg_flux, refs):
        """One nonlinear SSP-RK3 step (``main/timestep.py:141-187``): f advanced in place,
        ``elliptic`` left holding the field of stage s1, ``self.dt`` adapted from it."""
        if self.dt is None:
            raise ValueError("dt is not set (call adapt_time_step first, as main_loop does)")
        run = self._run(distribution, elliptic, grids, refs)
        st = self._host_state(run, float("inf"), 1)
        st.time = 0.0
        run.upload_state(st)
        run.launch(1, False)
        st = run.read_state()
        if st.status != 0:
            raise NonFiniteError("non-finite field or energy detected")
        self.dt = float(st.dt_next)
        elliptic.electric_field = _device.wrap(run.E.clone())
        elliptic.potential = _device.wrap(run.phi.clone())

    def ssp_rk_update(self, distribution, basis, grids, elliptic, dg_flux, refs):
        """One step of the linear SSP-RK stepper of any order (``main/timestep.py:189-229``),
        with the DG central-flux Poisson solve (``Elliptic.poisson``) for every stage field:
        acc = c0 f; copy <- copy + dt R(copy), acc += c_i copy (i = 1..order-1);
        f = acc + c_last dt R(copy); dt adapted from the last field.  Device kernels throughout
        (moment, ``vl_poisson_dg``, fused Euler stage, ``vl_axpby_interior``, RHS)."""
        if self.dt is None:
            raise ValueError("dt is not set (call adapt_time_step first)")
        c = [float(v) for v in np.asarray(self.coefficients).ravel()]
        f = _device.plain(distribution.arr)
        ctx = self._context(distribution, elliptic, grids, refs)
        key = (f.data_ptr(), tuple(f.shape), f.dtype)
        if getattr(self, "_lin_key", None) != key:
            self._lin = (torch.empty_like(f), torch.empty_like(f), torch.empty_like(f))
            self._lin_key = key
        A, B, R = self._lin
        stream = ctypes.c_void_p(_device.stream_handle())
        # periodic x ghosts of f; the copy (and the scratch) take all of f incl. ghosts
        ctx.sync_ghosts(f, A)
        ctx.sync_ghosts(f, B)
        _lib.call("vl_axpby_interior", ctx.handle, ctypes.c_void_p(f.data_ptr()), None, c[0], 0.0, stream)
        dt_t = torch.tensor([float(self.dt)], dtype=torch.float64, device=f.device)
        rho = torch.empty((grids.x.res, grids.x.order), dtype=torch.float64, device=f.device)

        def field(arr):
            ctx.moment(arr, rho)
            elliptic.poisson(charge_density=(rho.mean() - rho), grid=grids.x, basis=basis.b1)
            return _device.plain(elliptic.electric_field)

        for i in range(1, self.time_order):
            E = field(A)
            ctx.rk_stage(0, A, None, B, E, dt_t)          # B = A + dt R(A)
            A, B = B, A
            _lib.call("vl_axpby_interior", ctx.handle, ctypes.c_void_p(f.data_ptr()),
                      ctypes.c_void_p(A.data_ptr()), 1.0, c[i], stream)
        E = field(A)
        ctx.rhs(A, E, R, xhalo=_lib.VL_XHALO_PERIODIC)
        _lib.call("vl_axpby_interior", ctx.handle, ctypes.c_void_p(f.data_ptr()),
                  ctypes.c_void_p(R.data_ptr()), 1.0, c[-1] * float(self.dt), stream)
        self.adapt_time_step(max_speeds=get_max_speeds(grids, elliptic, refs),
                             dx=grids.x.dx, du=grids.u.dx, dv=grids.v.dx)

    def adapt_time_step(self, max_speeds, dx, du, dv):
        self.dt = self.courant / ((max_speeds[0] / dx) + (max_speeds[1] / du) + (max_speeds[2] / dv))


def get_max_speeds(grids, elliptic, refs):
    """Maximum characteristic speeds (``main/timestep.py:235-242``); one device->host read."""
    a = refs.electron_acceleration_multiplier
    E = _device.plain(elliptic.electric_field)
    emax = float(torch.amax(torch.abs(a * E)).item())
    return np.absolute(np.array([grids.u.arr_max,
                                 emax + abs(a * elliptic.magnetic_field * grids.v.arr_max),
                                 a * abs(elliptic.magnetic_field * grids.u.arr_max)]))
