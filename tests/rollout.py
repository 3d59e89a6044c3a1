"""Differentiable multi-step rollout for the tests: a torch.autograd.Function
over the library's fs_step / fs_step_adjoint (FP64 or FP32 contexts), with
binomial or uniform checkpointing of the step states.

Forward runs T steps keeping only the initial state.  Backward reverses the
steps with at most `snapshots` stored states besides the initial one: with s
snapshots and repetition number t, a segment of up to C(s+t, s) steps is
reversed by advancing to a split point m, taking a snapshot there, reversing
[m, end) with s-1 snapshots and then [start, m) with the same s snapshots
and repetition t-1 (Griewank's binomial schedule).  With a uniform schedule
(`every` = m) the forward keeps the states at steps 0, m, 2m, ... and each
segment is reversed by recomputing its states from its checkpoint.  The
adjoint fields of the context carry the bars from one reversed step to the
one before.

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


def _reverse_uniform(s, checkpoints, every, nsteps, dt, sched):
    """Reverse all steps segment by segment from the stored checkpoints."""
    for start in range(((nsteps - 1) // every) * every, -1, -every):
        end = min(start + every, nsteps)
        states = [checkpoints[start]]
        for _ in range(start + 1, end):
            states.append(_advance(s, states[-1], 1, dt, sched))
        sched.max_live_snapshots = max(sched.max_live_snapshots, len(checkpoints) + len(states))
        for st in reversed(states):
            _load(s, st)
            s.step_adjoint(dt)
            sched.adjoint_steps += 1


class Rollout(torch.autograd.Function):
    """phi(T), u(T), v(T), w(T) = rollout(phi0, u0, v0, w0, rho) over `nsteps`
    steps of length dt on the solver `s`, rho being the density of the phase
    `phase` ("pos" for phi > 0, "neg" for phi <= 0).  snapshots > 0: the
    binomial schedule with that many snapshots; every > 0: uniform
    checkpoints every `every` steps."""

    @staticmethod
    def forward(ctx, phi0, u0, v0, w0, rho, s, dt, nsteps, snapshots, sched, phase="pos", every=0):
        st0 = {k: t.detach().cpu().numpy().astype(np.float64) for k, t in zip(KEYS, (phi0, u0, v0, w0))}
        s.set_params(**{"rho_" + phase: float(rho.item())})
        ctx.checkpoints = {}
        if every > 0:
            st = st0
            for start in range(0, nsteps, every):
                ctx.checkpoints[start] = st
                st = _advance(s, st, min(every, nsteps - start), dt, sched)
            out = st
        else:
            out = _advance(s, st0, nsteps, dt, sched)
        ctx.s, ctx.dt, ctx.nsteps, ctx.snapshots, ctx.st0, ctx.sched = s, dt, nsteps, snapshots, st0, sched
        ctx.phase, ctx.every = phase, every
        return tuple(torch.from_numpy(out[k]) for k in KEYS)

    @staticmethod
    def backward(ctx, gphi, gu, gv, gw):
        s = ctx.s
        s.adjoint_reset()
        for k, g in zip(KEYS, (gphi, gu, gv, gw)):
            s.upload("adj_" + k, (g if g is not None else torch.zeros(s.shape(k), dtype=torch.float64)).numpy())
        if ctx.every > 0:
            _reverse_uniform(s, ctx.checkpoints, ctx.every, ctx.nsteps, ctx.dt, ctx.sched)
        else:
            _reverse(s, 0, ctx.nsteps, ctx.st0, ctx.snapshots, ctx.dt, ctx.sched)
        grads = [torch.from_numpy(s.download("adj_" + k)) for k in KEYS]
        bars = s.density_bars()
        rho_bar = torch.tensor(bars[1] if ctx.phase == "pos" else bars[0], dtype=torch.float64)
        return (*grads, rho_bar, None, None, None, None, None, None, None)
