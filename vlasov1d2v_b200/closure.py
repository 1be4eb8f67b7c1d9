"""Learned closure of the coarse velocity grid.

A coarse run (order 6, few velocity elements) misses the sub-grid velocity structure that a fine
run (order 8, 3x the elements per velocity axis) resolves.  The closure adds to the coarse RHS a
correction predicted per (x node, velocity element) by a small MLP from the element's nodal
patch and its neighbours' face traces, trained on fine runs of this solver:

    target = P R_fine(f_fine) - R_coarse(P f_fine),

P the L2 projection of the fine nodal state onto the coarse nodal space (per x element, and
3 x 3 fine velocity elements onto one coarse element).  Everything on the hot path is native:
feature extraction, the network's forward and backward passes (bf16 tensor cores, FP32
accumulation), Adam, and the application of the correction to each RK stage
(``vl_closure_features``, ``vl_mlp_*``, ``vl_closure_apply`` in ``include/vlasov1d2v.h``).
``ClosureStepper`` runs the coarse problem with the network; without a network (or after a
non-finite step) it is the plain coarse solver (the fallback).
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np
import scipy.special as sp
import torch

from . import _device, _lib
from .timestep import get_max_speeds

IN, HID, OUT, CN = 96, 128, 48, 6
NOUT = CN * CN


def _dims():
    a = [ctypes.c_int32() for _ in range(5)]
    _lib.call("vl_mlp_dims", *[ctypes.byref(x) for x in a])
    return [x.value for x in a]


def _vp(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    return ctypes.c_void_p(_device.stream_handle())


# ---------------------------------------------------------------------------------------------
# network parameters and training
# ---------------------------------------------------------------------------------------------
class MLP:
    """Device parameters of the closure network: FP32 master weights ([in][out] per layer,
    back to back) and biases, their bf16 copies in both layouts, and the Adam moments."""

    LAYERS = [(IN, HID), (HID, HID), (HID, HID), (HID, OUT)]

    def __init__(self, seed=0, device=None):
        dev = device or _device.device()
        _, _, _, nw, nb = _dims()
        rng = np.random.default_rng(seed)
        ws, bs = [], []
        for (k, n) in self.LAYERS:
            ws.append(rng.normal(0.0, math.sqrt(2.0 / k), size=(k, n)))
            bs.append(np.zeros(n))
        ws[-1] *= 0.1   # start near the plain solver
        self.master_w = torch.as_tensor(np.concatenate([w.ravel() for w in ws]), dtype=torch.float32, device=dev)
        self.master_b = torch.as_tensor(np.concatenate(bs), dtype=torch.float32, device=dev)
        assert self.master_w.numel() == nw and self.master_b.numel() == nb
        self.wf = torch.empty(nw, dtype=torch.bfloat16, device=dev)
        self.wb = torch.empty(nw, dtype=torch.bfloat16, device=dev)
        self.m_w, self.v_w = torch.zeros_like(self.master_w), torch.zeros_like(self.master_w)
        self.m_b, self.v_b = torch.zeros_like(self.master_b), torch.zeros_like(self.master_b)
        self.grad_w, self.grad_b = torch.zeros_like(self.master_w), torch.zeros_like(self.master_b)
        self.step = 0
        self.ymax = 1e30   # output clamp of the closure (set from the training targets)
        self.refresh_bf16()

    def layer_views(self, flat, transpose=False):
        out, off = [], 0
        for (k, n) in self.LAYERS:
            out.append(flat[off:off + k * n].view(n, k) if transpose else flat[off:off + k * n].view(k, n))
            off += k * n
        return out

    def refresh_bf16(self):
        """bf16 copies of the master weights in both layouts."""
        for src, dst_b, dst_f in zip(self.layer_views(self.master_w), self.layer_views(self.wb),
                                     self.layer_views(self.wf, transpose=True)):
            dst_b.copy_(src.to(torch.bfloat16))
            dst_f.copy_(src.t().to(torch.bfloat16))

    def forward(self, X, Y=None, save=None):
        n = X.shape[0]
        if Y is None:
            Y = torch.empty((n, OUT), dtype=torch.float32, device=X.device)
        H0 = Hh = Z = None
        if save is not None:
            H0, Hh, Z = save
        _lib.call("vl_mlp_forward", _vp(X), n, _vp(self.wf), _vp(self.wb), _vp(self.master_b), _vp(Y),
                  _vp(H0), _vp(Hh), _vp(Z), _stream())
        return Y

    def buffers(self, n, device):
        H0 = torch.empty((n, IN), dtype=torch.bfloat16, device=device)
        Hh = torch.empty((3, n, HID), dtype=torch.bfloat16, device=device)
        Z = torch.empty((3, n, HID), dtype=torch.float32, device=device)
        parts = torch.empty(int(_lib.load().vl_mlp_partial_floats(n)), dtype=torch.float32, device=device)
        Y = torch.empty((n, OUT), dtype=torch.float32, device=device)
        return {"H0": H0, "Hh": Hh, "Z": Z, "parts": parts, "Y": Y}

    def gradients(self, X, T, buf):
        """Forward + backward of the mean-squared loss on (X, T); gradients in grad_w / grad_b."""
        n = X.shape[0]
        self.forward(X, buf["Y"], (buf["H0"], buf["Hh"], buf["Z"]))
        _lib.call("vl_mlp_backward", _vp(buf["Y"]), _vp(T), n, T.shape[1], _vp(self.wf), _vp(self.wb),
                  _vp(self.master_b), _vp(buf["H0"]), _vp(buf["Hh"]), _vp(buf["Z"]), _vp(buf["parts"]),
                  _vp(self.grad_w), _vp(self.grad_b), _stream())
        return buf["Y"]

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        self.step += 1
        _lib.call("vl_mlp_adam", _vp(self.master_w), _vp(self.master_b), _vp(self.grad_w), _vp(self.grad_b),
                  _vp(self.m_w), _vp(self.v_w), _vp(self.m_b), _vp(self.v_b), _vp(self.wf), _vp(self.wb),
                  float(lr), float(beta1), float(beta2), float(eps), self.step, float(weight_decay), _stream())

    def state(self):
        return {"w": self.master_w.cpu().numpy(), "b": self.master_b.cpu().numpy()}

    def load(self, state):
        self.master_w.copy_(torch.as_tensor(state["w"]))
        self.master_b.copy_(torch.as_tensor(state["b"]))
        self.refresh_bf16()


def train(mlp, X, T, epochs=10, batch=8192, lr=2e-3, seed=0, val=None, log=None, noise=0.0,
          weight_decay=0.0):
    """Adam on shuffled minibatches (all on the device); ``noise`` adds Gaussian noise of that
    standard deviation to the state features of each minibatch (robustness of the closure to
    states off the training manifold).  Returns the loss history."""
    n = X.shape[0]
    g = torch.Generator(device=X.device)
    g.manual_seed(seed)
    buf = mlp.buffers(batch, X.device)
    hist = []
    steps_per_epoch = max(n // batch, 1)
    total = epochs * steps_per_epoch
    for ep in range(epochs):
        perm = torch.randperm(n, device=X.device, generator=g)
        tot = 0.0
        for s in range(steps_per_epoch):
            idx = perm[s * batch:(s + 1) * batch]
            xb, tb = X[idx].contiguous(), T[idx].contiguous()
            if noise > 0.0:
                xb[:, :84] += noise * torch.randn(xb[:, :84].shape, device=xb.device, generator=g)
            Y = mlp.gradients(xb, tb, buf)
            # cosine learning-rate decay
            k = ep * steps_per_epoch + s
            mlp.adam(lr * 0.5 * (1.0 + math.cos(math.pi * k / total)), weight_decay=weight_decay)
            if s % 16 == 0:
                tot += float(((Y[:, :NOUT] - tb) ** 2).mean())
        rec = {"epoch": ep, "train_loss": tot / max((steps_per_epoch + 15) // 16, 1)}
        if val is not None:
            rec["val_loss"] = evaluate(mlp, *val)
        hist.append(rec)
        if log:
            log(rec)
    return hist


def evaluate(mlp, X, T, batch=65536):
    tot, n = 0.0, X.shape[0]
    for s in range(0, n, batch):
        Y = mlp.forward(X[s:s + batch].contiguous())
        tot += float(((Y[:, :NOUT] - T[s:s + batch]) ** 2).sum())
    return tot / (n * NOUT)


# ---------------------------------------------------------------------------------------------
# fine -> coarse projection and training data
# ---------------------------------------------------------------------------------------------
def projection_1d(fine_nodes, coarse_nodes, ratio, nq=24):
    """P[nc, ratio * nf]: nodal values at the coarse nodes of the L2 projection (onto degree
    nc - 1) of the piecewise nodal polynomial on ``ratio`` equal sub-elements."""
    nf, nc = len(fine_nodes), len(coarse_nodes)
    xq, wq = np.polynomial.legendre.leggauss(nq)
    P = np.zeros((nc, ratio * nf))
    vc = np.array([sp.eval_legendre(s, coarse_nodes) for s in range(nc)])     # [s, coarse node]
    for q in range(ratio):
        lo, hi = -1.0 + 2.0 * q / ratio, -1.0 + 2.0 * (q + 1) / ratio
        xi = 0.5 * (hi - lo) * xq + 0.5 * (hi + lo)                         # coarse reference coords
        loc = xq                                                            # sub-element coords
        # fine Lagrange basis at the quadrature points
        ell = np.ones((nf, nq))
        for m in range(nf):
            for r in range(nf):
                if r != m:
                    ell[m] *= (loc - fine_nodes[r]) / (fine_nodes[m] - fine_nodes[r])
        for s in range(nc):
            ps = sp.eval_legendre(s, xi)
            coef = (2 * s + 1) / 2.0 * 0.5 * (hi - lo)
            P[:, q * nf:(q + 1) * nf] += np.outer(vc[s], coef * (ell * ps * wq).sum(axis=1))
    return P


class Projector:
    """L2 projection of fine states / RHS (order nf, ratio x velocity elements) to the coarse
    grid (order 6), on the device (FP64 tensor contractions)."""

    def __init__(self, fine_basis_nodes, coarse_basis_nodes, ratio=3, device=None):
        dev = device or _device.device()
        self.ratio = ratio
        self.px = torch.as_tensor(projection_1d(fine_basis_nodes, coarse_basis_nodes, 1), device=dev)
        self.pv = torch.as_tensor(projection_1d(fine_basis_nodes, coarse_basis_nodes, ratio), device=dev)

    def __call__(self, f):
        """Interior of a fine state [X, nf, U, nf, V, nf] -> coarse interior [nx, 6, nu/r, 6, nv/r, 6]."""
        t = _device.plain(f)[1:-1, :, 1:-1, :, 1:-1, :].double()
        nx, nf, nu, _, nv, _ = t.shape
        r = self.ratio
        t = t.reshape(nx, nf, nu // r, r * nf, nv // r, r * nf)
        return torch.einsum("pi,qj,sk,eiajbk->epaqbs", self.px, self.pv, self.pv, t)


def _field(ctx, f, nx, n):
    """E (and rho) of a state through the native moment + spectral Poisson solve."""
    rho = torch.empty((nx, n), dtype=torch.float64, device=f.device)
    ctx.moment(f, rho)
    E = torch.empty((nx + 2, n), dtype=torch.float64, device=f.device)
    ctx.poisson((rho.mean() - rho).contiguous(), E)
    return E


def features(coarse, f, E, escale):
    """Closure inputs (X [samples, 96], scale [samples]) of a coarse problem's state."""
    g = coarse.grids
    nx, nu, nv = g.x.res, g.u.res, g.v.res
    ns = nx * CN * nu * nv
    X = torch.empty((ns, IN), dtype=torch.float32, device=f.device)
    sc = torch.empty(ns, dtype=torch.float32, device=f.device)
    un = _device.const(g.u, "nodes", g.u.arr)
    vn = _device.const(g.v, "nodes", g.v.arr)
    prec = _lib.VL_FP64 if f.dtype == torch.float64 else _lib.VL_FP32
    _lib.call("vl_closure_features", _vp(f), prec, nx, nu, nv, _vp(E), float(coarse.refs.electron_acceleration_multiplier),
              float(coarse.elliptic.magnetic_field), _vp(un), _vp(vn), float(g.u.arr_max), float(g.v.arr_max),
              float(escale), _vp(X), _vp(sc), _stream())
    return X, sc


def correction_scale(coarse):
    """RHS / state scale of the coarse grid: umax J_u (used to make targets dimensionless)."""
    return float(coarse.grids.u.arr_max * coarse.grids.u.J)


def make_pair(fine, coarse, projector, escale):
    """One training snapshot: (X, T) of the current fine state (fine and coarse problems of the
    same physics; the coarse state's interior is overwritten with the projected fine state)."""
    from .context import get_context

    ff = _device.plain(fine.f.arr)
    cg, fg = coarse.grids, fine.grids
    fctx = get_context(fg, precision="fp64", accel=fine.refs.electron_acceleration_multiplier,
                       bfield=fine.elliptic.magnetic_field, kappa=fine.elliptic.poisson_coefficient)
    cctx = get_context(cg, precision="fp64", accel=coarse.refs.electron_acceleration_multiplier,
                       bfield=coarse.elliptic.magnetic_field, kappa=coarse.elliptic.poisson_coefficient)
    Ef = _field(fctx, ff, fg.x.res, fg.x.order)
    Rf = torch.empty_like(ff)
    fctx.rhs(ff, Ef, Rf, xhalo=_lib.VL_XHALO_PERIODIC)
    fc = _device.plain(coarse.f.arr)
    fc[1:-1, :, 1:-1, :, 1:-1, :] = projector(ff)
    fc[0] = fc[-2]
    fc[-1] = fc[1]
    Ec = _field(cctx, fc, cg.x.res, cg.x.order)
    Rc = torch.empty_like(fc)
    cctx.rhs(fc, Ec, Rc, xhalo=_lib.VL_XHALO_PERIODIC)
    target = projector(Rf) - Rc[1:-1, :, 1:-1, :, 1:-1, :]
    X, sc = features(coarse, fc, Ec, escale)
    # sample-major [e, i, a, b, j, k] / (scale * cscale)
    t = target.permute(0, 1, 2, 4, 3, 5).reshape(-1, NOUT)
    T = (t / (sc.double()[:, None] * correction_scale(coarse))).float()
    return X, T


# ---------------------------------------------------------------------------------------------
# coarse stepping with the closure
# ---------------------------------------------------------------------------------------------
_RK = [(None, None, 1.0), (3.0 / 4.0, 1.0 / 4.0, 1.0 / 4.0), (1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0)]


def runaway(times, energies, start, max_rate):
    """True when the field energies from index ``start`` on rise above the largest earlier one,
    W_max at t_max, by more than exp(2 max_rate (t_end - t_max)), t_end the last time."""
    past = energies[:start]
    i_max = max(range(len(past)), key=past.__getitem__)
    w0 = max(past[i_max], 1e-300)
    span = max(times[-1] - times[i_max], 1e-300)
    return max(energies[start:]) > w0 * math.exp(2.0 * max_rate * span)


class ClosureStepper:
    """Nonlinear SSP-RK3 on a coarse problem with the learned RHS correction after every stage;
    ``mlp=None`` runs the plain coarse operator through the same loop.  One step is a fixed
    sequence of device launches (native kernels + a few torch reductions), CUDA-graph captured."""

    def __init__(self, coarse, mlp=None, escale=1.0, alpha=1.0, constraint=None):
        """``alpha`` scales the learned correction (1: as trained; below 1: relaxed).
        ``constraint="charge"`` removes, per x node, the quadrature mean of the correction over
        velocity, so the closure cannot change the charge density that drives the field."""
        from .context import get_context

        self.p = coarse
        self.mlp = mlp
        self.escale = float(escale)
        self.alpha = float(alpha)
        if constraint not in (None, "charge"):
            raise ValueError("constraint must be None or 'charge'")
        self.mode = _lib.VL_CLOSURE_CHARGE if constraint == "charge" else _lib.VL_CLOSURE_PLAIN
        self._node_w = (ctypes.c_double * CN)(*[float(w) for w in coarse.basis.b1.weights])
        g = coarse.grids
        self.ctx = get_context(g, precision="fp64", accel=coarse.refs.electron_acceleration_multiplier,
                               bfield=coarse.elliptic.magnetic_field, kappa=coarse.elliptic.poisson_coefficient,
                               courant=coarse.stepper.courant)
        self.f = _device.plain(coarse.f.arr)
        dev = self.f.device
        self.sa, self.sb = torch.empty_like(self.f), torch.empty_like(self.f)
        self.ctx.sync_ghosts(self.f, self.sa)
        self.ctx.sync_ghosts(self.f, self.sb)
        self.nx, self.n = g.x.res, g.x.order
        self.E = torch.zeros((self.nx + 2, self.n), dtype=torch.float64, device=dev)
        self.rho = torch.empty((self.nx, self.n), dtype=torch.float64, device=dev)
        self.dt = torch.zeros(1, dtype=torch.float64, device=dev)
        self.energy = torch.zeros(1, dtype=torch.float64, device=dev)
        ns = self.nx * CN * g.u.res * g.v.res
        self.X = torch.empty((ns, IN), dtype=torch.float32, device=dev)
        self.sc = torch.empty(ns, dtype=torch.float32, device=dev)
        self.Y = torch.empty((ns, OUT), dtype=torch.float32, device=dev)
        self.cscale = correction_scale(coarse)
        self.un = _device.const(g.u, "nodes", g.u.arr)
        self.vn = _device.const(g.v, "nodes", g.v.arr)
        st = coarse.stepper
        st.adapt_time_step(get_max_speeds(g, coarse.elliptic, coarse.refs), g.x.dx, g.u.dx, g.v.dx)
        self.dt.fill_(st.dt)
        self.time = 0.0
        self.times, self.energies = [0.0], [float(coarse.elliptic.electric_energy(grid=g.x).get())]
        self._graph = None
        self._hist = None

    def _field(self, f):
        self.ctx.moment(f, self.rho)
        self.ctx.poisson((self.rho.mean() - self.rho).contiguous(), self.E)

    def _closure(self, inp, out, c2):
        if self.mlp is None:
            return
        g = self.p.grids
        _lib.call("vl_closure_features", _vp(inp), _lib.VL_FP64, self.nx, g.u.res, g.v.res, _vp(self.E),
                  float(self.p.refs.electron_acceleration_multiplier), float(self.p.elliptic.magnetic_field),
                  _vp(self.un), _vp(self.vn), float(g.u.arr_max), float(g.v.arr_max), self.escale,
                  _vp(self.X), _vp(self.sc), _stream())
        self.mlp.forward(self.X, self.Y)
        _lib.call("vl_closure_apply", _vp(out), _lib.VL_FP64, self.nx, g.u.res, g.v.res, _vp(self.Y),
                  _vp(self.sc), self.cscale, float(self.mlp.ymax), _vp(self.dt), float(c2 * self.alpha), None,
                  int(self.mode), ctypes.cast(self._node_w, ctypes.POINTER(ctypes.c_double)), _stream())

    def _step(self, k):
        f, sa, sb = self.f, self.sa, self.sb
        # periodic x ghosts of f (main/timestep.py:143)
        f[0].copy_(f[-2])
        f[-1].copy_(f[1])
        self._field(f)
        self.ctx.rk_stage(0, f, None, sa, self.E, self.dt)
        self._closure(f, sa, 1.0)
        self._field(sa)
        self.ctx.rk_stage(1, sa, f, sb, self.E, self.dt)
        self._closure(sa, sb, _RK[1][2])
        self._field(sb)
        # energy of E(s1) and the next dt (main/timestep.py:98-103, :184-185)
        _lib.call("vl_field_energy", self.ctx.handle, _vp(self.E), _vp(self._hist[0, k:k + 1]), _stream())
        _lib.call("vl_adapt_dt", self.ctx.handle, _vp(self.E), _vp(self._hist[1, k:k + 1]), _stream())
        self.ctx.rk_stage(2, sb, f, f, self.E, self.dt)
        self._closure(sb, f, _RK[2][2])
        self.dt.copy_(self._hist[1, k:k + 1])

    def run_steps(self, nsteps, batch=32, use_graph=True, max_rate=0.5):
        """Advance ``nsteps`` steps.  Fallback: a batch whose energy or dt is non-finite, or in
        which the field energy rises above its largest earlier value W_max by more than
        exp(2 max_rate (t - t_max)) (far above the physical growth rates of the cyclotron-harmonic
        instability; measured from the earlier maximum, not from the batch's first step, because
        the field energy oscillates through deep minima early in a run), is undone and the run
        continues with the plain coarse operator (``fallback_step`` records where)."""
        dev = self.f.device
        done = 0
        while done < nsteps:
            k = min(batch, nsteps - done)
            snap = (self.f.clone(), self.dt.clone(), self.time, len(self.times))
            try:
                self._batch(k, use_graph)
                bad = False
            except FloatingPointError:
                bad = True
            if not bad and self.mlp is not None:
                bad = runaway(self.times, self.energies, snap[3], max_rate)
            if bad:
                if self.mlp is None:
                    raise FloatingPointError("non-finite energy or dt in the plain coarse run")
                self.f.copy_(snap[0])
                self.dt.copy_(snap[1])
                self.time = snap[2]
                del self.times[snap[3]:]
                del self.energies[snap[3]:]
                self.mlp = None
                self.fallback_step = done
                self._graph = None
                self._hist = None
                continue
            done += k

    fallback_step = None

    def _batch(self, k, use_graph):
        dev = self.f.device
        if self._hist is None or self._hist.shape[1] != k or not use_graph:
            self._hist = torch.zeros((2, k), dtype=torch.float64, device=dev)
            self._graph = None
        if use_graph:
            if self._graph is None:
                for q in range(k):   # the first batch runs eagerly and warms the launch path
                    self._step(q)
                self._record(k)
                g = torch.cuda.CUDAGraph()
                s = torch.cuda.Stream()
                s.wait_stream(torch.cuda.current_stream())
                with torch.cuda.stream(s):
                    with torch.cuda.graph(g, stream=s):
                        for q in range(k):
                            self._step(q)
                torch.cuda.current_stream().wait_stream(s)
                # capture does not execute: the graph serves the next batches
                self._graph = g
                return
            self._graph.replay()
        else:
            for q in range(k):
                self._step(q)
        self._record(k)

    def _record(self, k):
        h = self._hist.cpu().numpy()
        for q in range(k):
            self.time += float(h[1, q])
            self.times.append(self.time)
            self.energies.append(float(h[0, q]))
        if not np.all(np.isfinite(h)):
            raise FloatingPointError("non-finite energy or dt in the closure run")


__all__ = ["MLP", "train", "evaluate", "Projector", "projection_1d", "make_pair", "features",
           "ClosureStepper", "correction_scale", "runaway"]
