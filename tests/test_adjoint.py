"""Adjoint tests through the C ABI (FP64 contexts on a B200).

1. Transpose (dot-product) tests per operator: for an operator F with
   inputs X and outputs Y, <Ybar, J dX> computed by central differences of
   the forward C-ABI operator must equal <Jt Ybar, dX> from the adjoint entry
   point, for random Ybar and dX (densities included where the operator
   depends on them).
2. The step adjoint against central finite differences of the FP64 oracle
   (oracle/fs_oracle.py, the CPU restatement of the reference step).
3. A multi-step rollout through torch.autograd with checkpointing, against
   finite differences of the plain FP64 GPU path.
"""
import numpy as np
import pytest

import fluid_simulator_backup_b200 as fs

pytestmark = pytest.mark.gpu

N = 12
FIELDS_VEL = ("u", "v", "w")


def shapes(n):
    return {"phi": (n, n, n), "u": (n, n, n + 1), "v": (n, n + 1, n), "w": (n + 1, n, n)}


def scene(n, seed, vel_scale=0.3):
    """A perturbed sphere level set and smooth, sign-changing velocities."""
    rng = np.random.default_rng(seed)
    x = (np.arange(n) + 0.5) / n
    X, Y, Z = x[None, None, :], x[None, :, None], x[:, None, None]
    phi = np.sqrt((X - 0.5) ** 2 + (Y - 0.42) ** 2 + (Z - 0.55) ** 2) - 0.27
    phi = phi + 0.01 * rng.standard_normal(phi.shape)
    xf = np.arange(n + 1) / n
    u = vel_scale * np.sin(2 * np.pi * (Y + 0.1)) * np.cos(np.pi * Z) + 0.05 * rng.standard_normal((n, n, n + 1))
    u = u * np.ones((n, n, n + 1))
    v = vel_scale * np.cos(2 * np.pi * (X + 0.2)) * np.ones((n, n + 1, n)) + 0.05 * rng.standard_normal((n, n + 1, n))
    w = vel_scale * np.sin(2 * np.pi * (Y + 0.3)) * np.ones((n + 1, n, n)) + 0.05 * rng.standard_normal((n + 1, n, n))
    del xf
    return {"phi": phi, "u": u, "v": v, "w": w}


def zero_walls(st):
    """The no-penetration zero on the wall faces of each component."""
    st = dict(st)
    u, v, w = st["u"].copy(), st["v"].copy(), st["w"].copy()
    u[:, :, 0] = u[:, :, -1] = 0.0
    v[:, 0, :] = v[:, -1, :] = 0.0
    w[0, :, :] = w[-1, :, :] = 0.0
    st.update(u=u, v=v, w=w)
    return st


def solver(n, **kw):
    p = dict(rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, tolerance=1e-13, stop=fs.FS_STOP_RELATIVE,
             max_iteration=100000, viscosity_tolerance=1e-14, viscosity_max_iteration=100000)
    p.update(kw)
    return fs.Solver(n, 1.0 / n, precision=fs.FS_PRECISION_FP64, **p)


def load(s, st, rho=None):
    for k in ("phi", "u", "v", "w"):
        s.upload(k, st[k])
    s.upload("pressure", np.zeros(s.shape("pressure")))
    if rho is not None:
        s.set_params(rho_neg=float(rho[0]), rho_pos=float(rho[1]))


def dot(a, b, keys):
    return sum(float(np.sum(a[k] * b[k])) for k in keys if k in a and k in b)


def transpose_check(s, forward, adjoint, X, dX, Ybar, out_keys, in_keys, h, rho=None, drho=None):
    """<Ybar, (F(X+h dX) - F(X-h dX)) / 2h>  vs  <Xbar, dX> (+ rho_bar . drho)."""
    def run(sign):
        st = {k: X[k] + sign * h * dX[k] if k in dX else X[k] for k in X}
        r = None if rho is None else np.array(rho) + (sign * h * np.array(drho) if drho is not None else 0.0)
        load(s, st, r)
        forward(s)
        return {k: s.download(k) for k in out_keys}
    yp, ym = run(+1), run(-1)
    jv = {k: (yp[k] - ym[k]) / (2 * h) for k in out_keys}
    lhs = dot(Ybar, jv, out_keys)
    load(s, X, rho)
    s.adjoint_reset()
    for k in out_keys:
        s.upload("adj_" + k, Ybar[k])
    adjoint(s)
    xbar = {k: s.download("adj_" + k) for k in in_keys}
    rhs = dot(xbar, dX, in_keys)
    if drho is not None:
        rb = s.density_bars()
        rhs += rb[0] * drho[0] + rb[1] * drho[1]
    return lhs, rhs


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


def rand_like(st, rng, keys):
    return {k: rng.standard_normal(st[k].shape) for k in keys}


def test_levelset_advection_adjoint_transpose():
    X = scene(N, 1)
    rng = np.random.default_rng(11)
    dX = rand_like(X, rng, ("phi", "u", "v", "w"))
    Ybar = rand_like(X, rng, ("phi",))
    dt = 0.2 / N
    with solver(N) as s:
        # WENO5 weights with eps = 1e-6 are very nonlinear where the smoothness
        # indicators vanish (linearly extrapolated ghosts, zero ghosts), so the
        # difference step must be small: at h = 1e-7 truncation is below 1e-7
        lhs, rhs = transpose_check(s, lambda s: s.advect_levelset(dt), lambda s: s.advect_levelset_adjoint(dt),
                                   X, dX, Ybar, ("phi",), ("phi", "u", "v", "w"), 1e-7)
    assert rel(lhs, rhs) < 1e-6, (lhs, rhs)


def test_velocity_advection_adjoint_transpose():
    X = scene(N, 2)
    rng = np.random.default_rng(12)
    dX = rand_like(X, rng, FIELDS_VEL)
    Ybar = rand_like(X, rng, FIELDS_VEL)
    dt = 0.2 / N
    with solver(N) as s:
        lhs, rhs = transpose_check(s, lambda s: s.advect_velocity(dt), lambda s: s.advect_velocity_adjoint(dt),
                                   X, dX, Ybar, FIELDS_VEL, FIELDS_VEL, 1e-7)
    assert rel(lhs, rhs) < 1e-6, (lhs, rhs)


@pytest.mark.parametrize("typo", [False, True])
def test_reinitialization_adjoint_transpose(typo):
    X = scene(N, 3)
    X["phi"] = X["phi"] * 1.3 + 0.02  # not a distance function: reinitialisation moves it
    rng = np.random.default_rng(13)
    dX = rand_like(X, rng, ("phi",))
    Ybar = rand_like(X, rng, ("phi",))
    with solver(N, flags=fs.FS_FLAG_REINIT_TYPO if typo else 0) as s:
        lhs, rhs = transpose_check(s, lambda s: s.reinitialize(), lambda s: s.reinitialize_adjoint(),
                                   X, dX, Ybar, ("phi",), ("phi",), 1e-7)
    assert rel(lhs, rhs) < 1e-5, (lhs, rhs)


def test_viscosity_adjoint_transpose():
    X = zero_walls(scene(N, 4))
    rng = np.random.default_rng(14)
    dX = zero_walls(rand_like(X, rng, ("phi", "u", "v", "w")))
    dX["phi"] = dX["phi"] * 0.01
    Ybar = rand_like(X, rng, FIELDS_VEL)
    dt = 0.5 / N
    rho, drho = (1.0, 1000.0), (0.3, 70.0)
    # viscosities large enough that the coefficients matter
    with solver(N, mu_neg=2e-2, mu_pos=5e-2) as s:
        lhs, rhs = transpose_check(s, lambda s: s.viscosity(dt), lambda s: s.viscosity_adjoint(dt),
                                   X, dX, Ybar, FIELDS_VEL, ("phi", "u", "v", "w"), 1e-5, rho, drho)
    assert rel(lhs, rhs) < 1e-6, (lhs, rhs)


def test_projection_adjoint_transpose():
    X = zero_walls(scene(N, 5))
    rng = np.random.default_rng(15)
    dX = rand_like(X, rng, ("phi", "u", "v", "w"))
    dX["phi"] = dX["phi"] * 0.01
    Ybar = rand_like(X, rng, FIELDS_VEL)
    dt = 0.5 / N
    rho, drho = (1.0, 1000.0), (0.3, 70.0)
    with solver(N) as s:
        lhs, rhs = transpose_check(s, lambda s: s.project(dt), lambda s: s.project_adjoint(dt),
                                   X, dX, Ybar, FIELDS_VEL, ("phi", "u", "v", "w"), 1e-5, rho, drho)
    assert rel(lhs, rhs) < 1e-6, (lhs, rhs)


@pytest.mark.parametrize("order", [1, 3])
def test_step_adjoint_transpose(order):
    n = 10
    X = zero_walls(scene(n, 6, vel_scale=0.2))
    rng = np.random.default_rng(16 + order)
    dX = zero_walls(rand_like(X, rng, ("phi", "u", "v", "w")))
    dX["phi"] = dX["phi"] * 0.01
    Ybar = rand_like(X, rng, ("phi", "u", "v", "w"))
    dt = 0.3 / n
    rho, drho = (1.0, 1000.0), (0.2, 50.0)
    with solver(n, order=order) as s:
        lhs, rhs = transpose_check(s, lambda s: s.step(dt), lambda s: s.step_adjoint(dt), X, dX, Ybar,
                                   ("phi", "u", "v", "w"), ("phi", "u", "v", "w"), 1e-6, rho, drho)
    assert rel(lhs, rhs) < 1e-5, (lhs, rhs)


def test_step_adjoint_matches_oracle_finite_differences():
    """Gradient of L = <Ybar, step(X)> w.r.t. the initial velocity and the
    water density, against central differences (h = 1e-6) of the FP64 CPU
    oracle of the reference step."""
    from oracle import fs_oracle as O
    n = 10
    dx = 1.0 / n
    X = zero_walls(scene(n, 7, vel_scale=0.2))
    rng = np.random.default_rng(27)
    Ybar = rand_like(X, rng, ("phi", "u", "v", "w"))
    dt = 0.3 / n
    P = dict(rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, gravity=(0.0, -9.8, 0.0), eps=1e-6,
             reinit_iterations=10, reinit_scaling=5, tol=1e-13, max_iter=100000, viscosity=True, visc_tol=1e-14)

    def loss_oracle(st, rho_pos):
        Q = dict(P, rho_pos=rho_pos)
        ph, uu, vv, ww, _, _ = O.step(st["phi"], st["u"], st["v"], st["w"], dx, dt, Q)
        out = {"phi": ph, "u": uu, "v": vv, "w": ww}
        return dot(Ybar, out, ("phi", "u", "v", "w"))

    with solver(n) as s:
        load(s, X)
        s.adjoint_reset()
        for k in ("phi", "u", "v", "w"):
            s.upload("adj_" + k, Ybar[k])
        s.step_adjoint(dt)
        grad = {k: s.download("adj_" + k) for k in ("phi", "u", "v", "w")}
        rho_bar = s.density_bars()
    h = 1e-6
    for d in range(3):
        dX = zero_walls(rand_like(X, np.random.default_rng(100 + d), FIELDS_VEL))
        dX = {k: dX[k] / np.sqrt(sum(np.sum(dX[q] ** 2) for q in FIELDS_VEL)) for k in FIELDS_VEL}
        plus = {k: X[k] + h * dX[k] if k in dX else X[k] for k in X}
        minus = {k: X[k] - h * dX[k] if k in dX else X[k] for k in X}
        fd = (loss_oracle(plus, 1000.0) - loss_oracle(minus, 1000.0)) / (2 * h)
        ad = dot(grad, dX, FIELDS_VEL)
        assert rel(fd, ad) < 1e-4, (d, fd, ad)
    # the density derivative is small against the loss: a step of 0.5 keeps
    # the solver-tolerance noise (1e-13 |L| / h) far below it
    hr = 0.5
    fd = (loss_oracle(X, 1000.0 + hr) - loss_oracle(X, 1000.0 - hr)) / (2 * hr)
    assert rel(fd, rho_bar[1]) < 1e-4, (fd, rho_bar)


def test_rollout_gradient_with_binomial_checkpointing():
    """Loss ||phi(T) - target||^2 after 6 steps, differentiated through the
    torch.autograd rollout (2 snapshots) and checked against central
    differences of the plain FP64 GPU forward."""
    import torch

    from rollout import Rollout, Schedule
    n, T, snaps = 10, 6, 2
    X = zero_walls(scene(n, 8, vel_scale=0.1))
    dt = 0.3 / n
    x = (np.arange(n) + 0.5) / n
    target = torch.from_numpy(np.broadcast_to(x[None, :, None] - 0.3, (n, n, n)).copy())
    with solver(n) as s:
        ts = {k: torch.tensor(X[k], requires_grad=True) for k in ("phi", "u", "v", "w")}
        rho = torch.tensor(1000.0, dtype=torch.float64, requires_grad=True)
        sched = Schedule()
        out = Rollout.apply(ts["phi"], ts["u"], ts["v"], ts["w"], rho, s, dt, T, snaps, sched)
        loss = torch.sum((out[0] - target) ** 2)
        loss.backward()
        assert sched.adjoint_steps == T
        assert sched.max_live_snapshots <= snaps
        grad = {k: ts[k].grad.numpy() for k in ("u", "v", "w")}
        g_rho = float(rho.grad)

        def loss_fd(st, rho_pos):
            s.set_params(rho_pos=rho_pos)
            load(s, st)
            for _ in range(T):
                s.step(dt)
            return float(np.sum((s.download("phi") - target.numpy()) ** 2))

        h = 1e-6
        for d in range(3):
            dX = zero_walls(rand_like(X, np.random.default_rng(200 + d), FIELDS_VEL))
            plus = {k: X[k] + h * dX[k] if k in dX else X[k] for k in X}
            minus = {k: X[k] - h * dX[k] if k in dX else X[k] for k in X}
            fd = (loss_fd(plus, 1000.0) - loss_fd(minus, 1000.0)) / (2 * h)
            ad = dot(grad, dX, FIELDS_VEL)
            assert rel(fd, ad) < 1e-4, (d, fd, ad)
        hr = 0.5
        fd = (loss_fd(X, 1000.0 + hr) - loss_fd(X, 1000.0 - hr)) / (2 * hr)
        assert rel(fd, g_rho) < 1e-3, (fd, g_rho)
