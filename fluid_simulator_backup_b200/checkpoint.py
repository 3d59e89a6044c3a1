"""Reversal of a multi-step rollout with bounded memory: the adjoint of T
steps from the states of a few checkpoints, recomputing the rest.

The library's fs_step_adjoint differentiates ONE step from its input state
(it recomputes that step's forward with a tape).  Differentiating T steps
needs the input state of every step in reverse order; keeping all of them
costs T states, recomputing each from the start costs T^2/2 steps.  Two
schedules are provided:

- binomial (Griewank's revolve): with s snapshots and repetition number t a
  segment of up to C(s+t, s) steps is reversed by advancing to a split
  point m, taking a snapshot there, reversing [m, end) with s-1 snapshots
  and then [start, m) with the same s snapshots and repetition t-1;
- uniform: checkpoints every m steps kept from the forward pass, each
  segment reversed by recomputing its states from its checkpoint.

States are host copies (FP64 arrays) of phi, u, v, w.  The context's
adjoint fields carry the bars from one reversed step to the one before: on
entry they hold the bars of the final state, on return the bars of the
initial state, with the density bars accumulated in the context.
"""
from math import comb

KEYS = ("phi", "u", "v", "w")


class Schedule:
    """Counts of the work a reversal did."""

    def __init__(self):
        self.forward_steps = 0
        self.adjoint_steps = 0
        self.max_live_snapshots = 0
        self.live = 0


def load(s, st):
    for k in KEYS:
        s.upload(k, st[k])


def save(s):
    return {k: s.download(k) for k in KEYS}


def advance(s, st, nsteps, dt, sched):
    """The state after nsteps steps from st."""
    load(s, st)
    for _ in range(nsteps):
        s.step(dt)
        sched.forward_steps += 1
    return save(s)


def _repetition(n, snaps):
    t = 0
    while comb(snaps + t, snaps) < n:
        t += 1
    return t


def reverse_binomial(s, a, b, st_a, snaps, dt, sched):
    """Reverse steps [a, b) given the state before step a; bars of the state
    after step b-1 are in the context's adjoint fields on entry, those of
    the state before step a on return."""
    n = b - a
    if n <= 0:
        return
    if n == 1:
        load(s, st_a)
        s.step_adjoint(dt)
        sched.adjoint_steps += 1
        return
    if snaps == 0:
        for k in range(b - 1, a - 1, -1):
            st_k = advance(s, st_a, k - a, dt, sched)
            load(s, st_k)
            s.step_adjoint(dt)
            sched.adjoint_steps += 1
        return
    t = _repetition(n, snaps)
    right = min(n - 1, comb(snaps - 1 + t, snaps - 1))  # steps reversed with one snapshot fewer
    m = b - right
    st_m = advance(s, st_a, m - a, dt, sched)
    sched.live += 1
    sched.max_live_snapshots = max(sched.max_live_snapshots, sched.live)
    reverse_binomial(s, m, b, st_m, snaps - 1, dt, sched)
    sched.live -= 1
    del st_m
    reverse_binomial(s, a, m, st_a, snaps, dt, sched)


def forward_uniform(s, st0, nsteps, every, dt, sched):
    """The forward pass keeping checkpoints every `every` steps; returns
    (final state, checkpoints {step: state})."""
    checkpoints = {}
    st = st0
    for start in range(0, nsteps, every):
        checkpoints[start] = st
        st = advance(s, st, min(every, nsteps - start), dt, sched)
    return st, checkpoints


def reverse_uniform(s, checkpoints, every, nsteps, dt, sched):
    """Reverse all steps segment by segment from the stored checkpoints."""
    for start in range(((nsteps - 1) // every) * every, -1, -every):
        end = min(start + every, nsteps)
        states = [checkpoints[start]]
        for _ in range(start + 1, end):
            states.append(advance(s, states[-1], 1, dt, sched))
        sched.max_live_snapshots = max(sched.max_live_snapshots, len(checkpoints) + len(states))
        for st in reversed(states):
            load(s, st)
            s.step_adjoint(dt)
            sched.adjoint_steps += 1
