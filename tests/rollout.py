"""Differentiable multi-step rollout for the tests: a torch.autograd.Function
over the library's fs_step / fs_step_adjoint (FP64 contexts), with binomial
checkpointing of the step states.

Forward runs T steps keeping only the initial state.  Backward reverses the
steps with at most `snapshots` stored states besides the initial one: with s
snapshots and repetition number t, a segment of up to C(s+t, s) steps is
reversed by advancing to a split point m, taking a snapshot there, reversing
[m, end) with s-1 snapshots and then [start, m) with the same s snapshots
and repetition t-1 (Griewank's binomial schedule).  The adjoint fields of the
context carry the bars from one reversed step to the one before.

Test infrastructure only: the library itself knows nothing of torch.
"""
from math import comb

import numpy as np
import torch

KEYS = ("phi", "u", "v", "w")


def _load(s, st):
    for k in KEYS:
        s.upload(k, st[k])


def _save(s):
    return {k: s.download(k) for k in KEYS}


class Schedule:
    """Counts of the work a reversal did (for the tests' memory/recompute checks)."""

    def __init__(self):
        self.forward_steps = 0
        self.adjoint_steps = 0
        self.max_live_snapshots = 0
        self.live = 0


def _advance(s, st, nsteps, dt, sched):
    _load(s, st)
    for _ in range(nsteps):
        s.step(dt)
        sched.forward_steps += 1
    return _save(s)


def _repetition(n, snaps):
    t = 0
    while comb(snaps + t, snaps) < n:
        t += 1
    return t


def _reverse(s, a, b, st_a, snaps, dt, sched):
    """Bars of the state after step b-1 are in the context's adjoint fields on
    entry; on return they are the bars of the state before step a."""
    n = b - a
    if n == 1:
        _load(s, st_a)
        s.step_adjoint(dt)
        sched.adjoint_steps += 1
        return
    if snaps == 0:
        for k in range(b - 1, a - 1, -1):
            st_k = _advance(s, st_a, k - a, dt, sched)
            _load(s, st_k)
            s.step_adjoint(dt)
            sched.adjoint_steps += 1
        return
    t = _repetition(n, snaps)
    right = min(n - 1, comb(snaps - 1 + t, snaps - 1))  # steps reversed with one snapshot fewer
    m = b - right
    st_m = _advance(s, st_a, m - a, dt, sched)
    sched.live += 1
    sched.max_live_snapshots = max(sched.max_live_snapshots, sched.live)
    _reverse(s, m, b, st_m, snaps - 1, dt, sched)
    sched.live -= 1
    del st_m
    _reverse(s, a, m, st_a, snaps, dt, sched)


class Rollout(torch.autograd.Function):
    """phi(T), u(T), v(T), w(T) = rollout(phi0, u0, v0, w0, rho_pos) over
    `nsteps` steps of length dt on the FP64 solver `s`."""

    @staticmethod
    def forward(ctx, phi0, u0, v0, w0, rho_pos, s, dt, nsteps, snapshots, sched):
        st0 = {k: t.detach().cpu().numpy().astype(np.float64) for k, t in zip(KEYS, (phi0, u0, v0, w0))}
        s.set_params(rho_pos=float(rho_pos.item()))
        out = _advance(s, st0, nsteps, dt, sched)
        ctx.s, ctx.dt, ctx.nsteps, ctx.snapshots, ctx.st0, ctx.sched = s, dt, nsteps, snapshots, st0, sched
        return tuple(torch.from_numpy(out[k]) for k in KEYS)

    @staticmethod
    def backward(ctx, gphi, gu, gv, gw):
        s = ctx.s
        s.adjoint_reset()
        for k, g in zip(KEYS, (gphi, gu, gv, gw)):
            s.upload("adj_" + k, (g if g is not None else torch.zeros(s.shape(k), dtype=torch.float64)).numpy())
        _reverse(s, 0, ctx.nsteps, ctx.st0, ctx.snapshots, ctx.dt, ctx.sched)
        grads = [torch.from_numpy(s.download("adj_" + k)) for k in KEYS]
        rho_bar = torch.tensor(s.density_bars()[1], dtype=torch.float64)
        return (*grads, rho_bar, None, None, None, None, None)
