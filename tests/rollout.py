"""Differentiable multi-step rollout for the tests: a torch.autograd.Function
over the library's fs_step / fs_step_adjoint (FP64 or FP32 contexts), with
binomial or uniform checkpointing of the step states (the schedules of
fluid_simulator_backup_b200.checkpoint).

Forward runs T steps keeping only the initial state (binomial) or the states
at steps 0, m, 2m, ... (uniform).  Backward reverses the steps with the
chosen schedule; the adjoint fields of the context carry the bars from one
reversed step to the one before.

Test infrastructure only: the library itself knows nothing of torch.
"""
import numpy as np
import torch

from fluid_simulator_backup_b200.checkpoint import (KEYS, Schedule, advance, forward_uniform, reverse_binomial,
                                                    reverse_uniform)


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
            out, ctx.checkpoints = forward_uniform(s, st0, nsteps, every, dt, sched)
        else:
            out = advance(s, st0, nsteps, dt, sched)
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
            reverse_uniform(s, ctx.checkpoints, ctx.every, ctx.nsteps, ctx.dt, ctx.sched)
        else:
            reverse_binomial(s, 0, ctx.nsteps, ctx.st0, ctx.snapshots, ctx.dt, ctx.sched)
        grads = [torch.from_numpy(s.download("adj_" + k)) for k in KEYS]
        bars = s.density_bars()
        rho_bar = torch.tensor(bars[1] if ctx.phase == "pos" else bars[0], dtype=torch.float64)
        return (*grads, rho_bar, None, None, None, None, None, None, None)
