"""The rollout reversal schedules (binomial and uniform checkpointing) on a
host-side stand-in for a solver context: a nonlinear map per step whose
adjoint must be evaluated at each step's own input state.  Checks the
gradient against the directly accumulated chain rule, the order of the
reversed steps, the snapshot bound and the recompute count of the binomial
schedule (Griewank's optimum for s snapshots)."""
from math import comb

import numpy as np
import pytest

from fluid_simulator_backup_b200 import checkpoint as ck


class FakeSolver:
    """step: x <- x + dt sin(x) + 0.1 dt (u, v, w mixed in); step_adjoint: the
    transposed Jacobian at the state loaded before the call."""

    def __init__(self, n=5):
        self.f = {k: np.zeros(n) for k in ck.KEYS}
        self.a = {k: np.zeros(n) for k in ck.KEYS}
        self.t = 0
        self.reversed = []

    def upload(self, k, a):
        (self.a if k.startswith("adj_") else self.f)[k.replace("adj_", "")] = np.array(a, dtype=np.float64)

    def download(self, k):
        return (self.a if k.startswith("adj_") else self.f)[k.replace("adj_", "")].copy()

    def _step(self, f, dt):
        g = dict(f)
        g["phi"] = f["phi"] + dt * np.sin(f["phi"]) + 0.1 * dt * f["u"]
        g["u"] = f["u"] + dt * np.cos(f["v"])
        g["v"] = f["v"] * (1.0 + dt * f["w"])
        g["w"] = f["w"]
        return g

    def step(self, dt):
        self.f = self._step(self.f, dt)

    def step_adjoint(self, dt):
        f, a = self.f, self.a
        b = {k: np.zeros_like(a[k]) for k in ck.KEYS}
        b["phi"] += a["phi"] * (1.0 + dt * np.cos(f["phi"]))
        b["u"] += a["phi"] * 0.1 * dt + a["u"]
        b["v"] += -a["u"] * dt * np.sin(f["v"]) + a["v"] * (1.0 + dt * f["w"])
        b["w"] += a["v"] * dt * f["v"] + a["w"]
        self.a = b
        self.reversed.append(self.f["phi"][0])
        self.f = self._step(f, dt)  # the schedules must not rely on the fields after an adjoint step


def chain_rule(st0, nsteps, dt, bar):
    s = FakeSolver(len(st0["phi"]))
    states = [st0]
    for _ in range(nsteps):
        states.append(s._step(states[-1], dt))
    for st in reversed(states[:-1]):
        s.f, s.a = dict(st), bar
        s.step_adjoint(dt)
        bar = s.a
    return bar, [st["phi"][0] for st in reversed(states[:-1])]


@pytest.mark.parametrize("nsteps,snaps", [(1, 1), (7, 0), (10, 2), (16, 3), (35, 3), (40, 4)])
def test_binomial_matches_chain_rule(nsteps, snaps):
    rng = np.random.default_rng(nsteps)
    st0 = {k: rng.normal(size=5) for k in ck.KEYS}
    bar0 = {k: rng.normal(size=5) for k in ck.KEYS}
    dt = 0.05
    s = FakeSolver()
    for k in ck.KEYS:
        s.upload("adj_" + k, bar0[k])
    sched = ck.Schedule()
    ck.reverse_binomial(s, 0, nsteps, st0, snaps, dt, sched)
    want, order = chain_rule(st0, nsteps, dt, bar0)
    for k in ck.KEYS:
        np.testing.assert_allclose(s.a[k], want[k], rtol=1e-13, atol=1e-13)
    assert np.allclose(s.reversed, order, rtol=0, atol=0)
    assert sched.adjoint_steps == nsteps
    assert sched.max_live_snapshots <= snaps
    if snaps > 0 and nsteps > 1:
        t = ck._repetition(nsteps, snaps)
        assert nsteps <= comb(snaps + t, snaps)
        # Griewank: at most t * nsteps forward steps for the reversal
        assert sched.forward_steps <= t * nsteps


@pytest.mark.parametrize("nsteps,every", [(8, 8), (32, 8), (13, 4), (5, 1)])
def test_uniform_matches_chain_rule(nsteps, every):
    rng = np.random.default_rng(100 + nsteps)
    st0 = {k: rng.normal(size=5) for k in ck.KEYS}
    bar0 = {k: rng.normal(size=5) for k in ck.KEYS}
    dt = 0.05
    s = FakeSolver()
    sched = ck.Schedule()
    out, cps = ck.forward_uniform(s, st0, nsteps, every, dt, sched)
    assert sorted(cps) == list(range(0, nsteps, every))
    direct = st0
    for _ in range(nsteps):
        direct = s._step(direct, dt)
    for k in ck.KEYS:
        np.testing.assert_allclose(out[k], direct[k], rtol=1e-14)
    for k in ck.KEYS:
        s.upload("adj_" + k, bar0[k])
    ck.reverse_uniform(s, cps, every, nsteps, dt, sched)
    want, order = chain_rule(st0, nsteps, dt, bar0)
    for k in ck.KEYS:
        np.testing.assert_allclose(s.a[k], want[k], rtol=1e-13, atol=1e-13)
    assert np.allclose(s.reversed, order, rtol=0, atol=0)
    assert sched.adjoint_steps == nsteps
    assert sched.forward_steps == nsteps + sum(min(every, nsteps - a) - 1 for a in range(0, nsteps, every))
