"""Gradients through the small step (1D, m0 = 0, FP64): the C ABI's
oshun_adjoint_* entry points wrapped as a torch.autograd.Function with RK-step
checkpointing.

    run = Run(cfg)                        # one oshun_adjoint handle
    Q = StepsWithCheckpoints.apply(y0, run, nsteps, every, weight)
    Q.backward()                          # y0.grad

The forward keeps the state every `every` steps; the backward walks the
segments from the last, recomputes the states of a segment from its
checkpoint and applies the step transposes (oshun_adjoint_vjp) in reverse.
The loss is the time integral sum_n dt <weight, y_n> over the states after
steps 1..nsteps (any linear functional of the state; the heat flux of one
cell in the tests and the benchmark's sensitivity case).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from .abi import OshunError, load, make_cfg


class Run:
    """One oshun_adjoint handle.  Called on a torch stream other than the
    default one, the handle's calls are queued on that same stream and do not
    wait (the torch operations around them are ordered by the stream); on the
    default stream every call waits for torch's work first and returns
    synchronized."""

    def __init__(self, **cfg):
        self.lib = load()
        self.cfg = make_cfg(**cfg)
        self._a = ctypes.c_void_p()
        self._check(self.lib.oshun_adjoint_create(ctypes.byref(self.cfg), ctypes.byref(self._a)),
                    "oshun_adjoint_create")
        n = ctypes.c_longlong()
        self._check(self.lib.oshun_adjoint_state_size(self._a, ctypes.byref(n)), "oshun_adjoint_state_size")
        self.n = n.value
        self.dt = self.cfg.dt
        self._stream = 0   # the torch stream the handle's calls are queued on (0: none, they wait)

    def _check(self, rc, what):
        if rc != 0:
            raise OshunError(rc, what, self.lib.oshun_last_error().decode())

    def close(self):
        if self._a:
            self.lib.oshun_adjoint_destroy(self._a)
            self._a = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _order(self):
        """Queue the handle's calls on torch's current stream when it is not
        the default stream; otherwise wait for torch's work (the calls wait too)."""
        cur = torch.cuda.current_stream()
        if cur.cuda_stream != self._stream:
            self._check(self.lib.oshun_adjoint_set_stream(self._a, ctypes.c_void_p(cur.cuda_stream or None)),
                        "oshun_adjoint_set_stream")
            self._stream = cur.cuda_stream
        if self._stream == 0:
            cur.synchronize()

    def forward(self, y: torch.Tensor, clocks, collisions: bool = True) -> torch.Tensor:
        out = torch.empty_like(y)
        self._order()
        self._check(self.lib.oshun_adjoint_forward(self._a, y.data_ptr(), out.data_ptr(), int(collisions), *clocks),
                    "oshun_adjoint_forward")
        return out

    def vjp(self, y: torch.Tensor, lam_next: torch.Tensor, clocks, collisions: bool = True) -> torch.Tensor:
        lam = torch.empty_like(y)
        lam_next = lam_next.contiguous()
        self._order()
        self._check(self.lib.oshun_adjoint_vjp(self._a, y.data_ptr(), lam_next.data_ptr(),
                                               lam.data_ptr(), int(collisions), *clocks), "oshun_adjoint_vjp")
        return lam

    def clocks(self, nsteps: int, collisions: bool = True):
        """(t, t_ee, t_eb) before each step, by the reference's clock arithmetic"""
        t = t_ee = t_eb = self.cfg.t0
        out = []
        for _ in range(nsteps):
            out.append((t, t_ee, t_eb))
            t += self.dt
            if collisions:
                t_ee = t_eb = t
        return out


class StepsWithCheckpoints(torch.autograd.Function):
    """Q = sum_{n=1..N} dt <weight, y_n>, y_n = step^n(y0), FP64 device vectors
    in the plane layout; the state is kept every `every` steps."""

    @staticmethod
    def forward(ctx, y0, run: Run, nsteps: int, every: int, weight, collisions: bool = True):
        clocks = run.clocks(nsteps, collisions)
        ckpt = {0: y0.detach().clone()}
        y = y0.detach()
        Q = torch.zeros((), dtype=torch.float64, device=y0.device)
        for n in range(nsteps):
            y = run.forward(y, clocks[n], collisions)
            Q = Q + run.dt * torch.dot(weight, y)
            if (n + 1) % every == 0 and n + 1 < nsteps:
                ckpt[n + 1] = y.clone()
        ctx.run, ctx.nsteps, ctx.every, ctx.collisions = run, nsteps, every, collisions
        ctx.clocks, ctx.ckpt = clocks, ckpt
        ctx.save_for_backward(weight)
        return Q

    @staticmethod
    def backward(ctx, gQ):
        (weight,) = ctx.saved_tensors
        run, nsteps, every = ctx.run, ctx.nsteps, ctx.every
        lam = torch.zeros_like(weight)
        starts = sorted(ctx.ckpt)
        for k in reversed(range(len(starts))):
            n0 = starts[k]
            n1 = starts[k + 1] if k + 1 < len(starts) else nsteps
            # recompute the states of this segment from its checkpoint
            states = [ctx.ckpt[n0]]
            for n in range(n0, n1 - 1):
                states.append(run.forward(states[-1], ctx.clocks[n], ctx.collisions))
            for n in reversed(range(n0, n1)):
                lam = lam + gQ * run.dt * weight          # the loss term of y_{n+1}
                lam = run.vjp(states[n - n0], lam, ctx.clocks[n], ctx.collisions)
        return lam, None, None, None, None, None


def state_layout(cfg) -> dict:
    """slices of the plane-layout vector: f (l0+1, nx, np), fields (6, nx)"""
    nx, np_, l0 = cfg["numx"], cfg["nump"], cfg["l0"]
    fsz = (l0 + 1) * nx * np_
    return dict(f=slice(0, fsz), fields=slice(fsz, fsz + 6 * nx), fshape=(l0 + 1, nx, np_), n=fsz + 6 * nx)


def heat_flux_weight(cfg, cell: int, device="cuda") -> torch.Tensor:
    """weight of q(cell) = (4 pi / 3) int p^2 v (gamma - 1) f_10 dp (trapezoid in
    p): the energy flux carried by f_10 at one cell, as a plane-layout vector"""
    lay = state_layout(cfg)
    np_, nx = cfg["nump"], cfg["numx"]
    p = np.arange(np_) * ((cfg["pmax"] - cfg["pmin"]) / (np_ - 1)) + cfg["pmin"]
    g = np.sqrt(1 + p * p)
    w = 4 * np.pi / 3 * p ** 2 * (p / g) * (g - 1)
    tr = np.full(np_, p[1] - p[0])
    tr[0] *= 0.5
    tr[-1] *= 0.5
    wv = np.zeros(lay["n"])
    wv[(1 * nx + cell) * np_:(1 * nx + cell + 1) * np_] = w * tr
    return torch.tensor(wv, dtype=torch.float64, device=device)
