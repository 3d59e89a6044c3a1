"""Adjoints over FP32 states with FP64 bars and reductions, and the
differentiable dam break of the 96^3 configuration.

- One step: the adjoint of an FP32 + FP64 refinement context (forward states
  and tape in FP32, every bar, derivative and sum in FP64) against the FP64
  context's adjoint from the same state.
- The 96^3 dam break over 32 steps: seeded N(0, 0.05^2) face velocities, loss
  L = ||phi(T) - (y - 0.3)||_2^2, gradient w.r.t. the initial velocity (three
  face arrays) and the density ratio (water density, air fixed at 1) through
  the torch.autograd rollout with checkpoints every 8 steps, in FP32 (the
  configuration's precision) and in FP64; checked against central
  differences (h = 1e-6) of the plain FP64 GPU forward in 16 unit directions
  drawn with default_rng(1..16)."""
import numpy as np
import pytest

import fluid_simulator_backup_b200 as fs

pytestmark = pytest.mark.gpu

KEYS = ("phi", "u", "v", "w")
VEL = ("u", "v", "w")


def dam_break(n):
    x = (np.arange(n) + 0.5) / n
    X, Y, Z = x[None, None, :], x[None, :, None], x[:, None, None]
    lo, hi = np.array([0.0, 0.0, 0.0]), np.array([0.4, 0.6, 1.0])
    d = [np.maximum(lo[a] - c, c - hi[a]) for a, c in enumerate((X, Y, Z))]
    d = np.broadcast_arrays(*d)
    outside = np.sqrt(sum(np.maximum(q, 0.0) ** 2 for q in d))
    inside = np.minimum(np.maximum(np.maximum(d[0], d[1]), d[2]), 0.0)
    return outside + inside


def zero_walls(st):
    out = dict(st)
    out["u"] = out["u"].copy(); out["u"][:, :, 0] = 0.0; out["u"][:, :, -1] = 0.0
    out["v"] = out["v"].copy(); out["v"][:, 0, :] = 0.0; out["v"][:, -1, :] = 0.0
    out["w"] = out["w"].copy(); out["w"][0] = 0.0; out["w"][-1] = 0.0
    return out


def initial_state(n):
    """phi0 the dam break; u0 ~ N(0, 0.05^2) on every face, drawn with
    default_rng(0) in (component, k, j, i) order (wall faces then held at
    zero, as the step's no-penetration condition does)."""
    rng = np.random.default_rng(0)
    st = {"phi": dam_break(n),
          "u": rng.normal(0.0, 0.05, size=(n, n, n + 1)),
          "v": rng.normal(0.0, 0.05, size=(n, n + 1, n)),
          "w": rng.normal(0.0, 0.05, size=(n + 1, n, n))}
    return zero_walls(st)


def params(precision, tol):
    return dict(rho_neg=1000.0, rho_pos=1.0, mu_neg=1e-3, mu_pos=1.8e-5, precision=precision, tolerance=tol,
                stop=fs.FS_STOP_RELATIVE, max_iteration=40000, order=3, viscosity=1, viscosity_tolerance=1e-12,
                viscosity_max_iteration=4000, reinit_iterations=10, reinit_scaling=5)


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def test_fp32_step_adjoint_matches_fp64_adjoint():
    """Same state and output bars: the FP32-state adjoint against the FP64
    one; they differ by the FP32 rounding of the forward states the
    derivatives are evaluated at."""
    n = 14
    rng = np.random.default_rng(3)
    X = initial_state(n)
    X["phi"] = X["phi"] + 0.01 * rng.normal(size=X["phi"].shape)
    Ybar = {k: rng.normal(size=X[k].shape) for k in KEYS}
    dt = 0.3 / n
    out = {}
    for precision in (fs.FS_PRECISION_FP64, fs.FS_PRECISION_FP32_REFINE):
        with fs.Solver(n, 1.0 / n, **params(precision, 1e-11)) as s:
            for k in KEYS:
                s.upload(k, X[k])
            s.adjoint_reset()
            for k in KEYS:
                s.upload("adj_" + k, Ybar[k])
            s.step_adjoint(dt)
            out[precision] = ({k: s.download("adj_" + k) for k in KEYS}, s.density_bars())
    (g64, r64), (g32, r32) = out[fs.FS_PRECISION_FP64], out[fs.FS_PRECISION_FP32_REFINE]
    for k in KEYS:
        err = np.linalg.norm(g32[k] - g64[k]) / np.linalg.norm(g64[k])
        print(f"FP32-state adjoint vs FP64, bar of {k}: {err:.2e}")
        assert err < 1e-3, (k, err)
    # the two density bars differ by three orders of magnitude here (the water
    # density's derivative is a small difference of large terms), so both are
    # compared on the scale of the larger one
    scale = max(abs(r64[0]), abs(r64[1]))
    print(f"density bars FP32 {r32}, FP64 {r64}")
    assert abs(r32[0] - r64[0]) < 1e-3 * scale and abs(r32[1] - r64[1]) < 1e-3 * scale


def test_differentiable_dam_break_96_32_steps():
    import torch

    from rollout import Rollout, Schedule
    n, T, every = 96, 32, 8
    dx = 1.0 / n
    dt = 2e-3
    X = initial_state(n)
    y = (np.arange(n) + 0.5) / n
    target = np.broadcast_to(y[None, :, None] - 0.3, (n, n, n)).copy()
    grads = {}
    for precision, tol in ((fs.FS_PRECISION_FP32_REFINE, 1e-11), (fs.FS_PRECISION_FP64, 1e-11)):
        with fs.Solver(n, dx, **params(precision, tol)) as s:
            ts = {k: torch.tensor(X[k], requires_grad=True) for k in KEYS}
            rho = torch.tensor(1000.0, dtype=torch.float64, requires_grad=True)
            sched = Schedule()
            out = Rollout.apply(ts["phi"], ts["u"], ts["v"], ts["w"], rho, s, dt, T, 0, sched, "neg", every)
            loss = torch.sum((out[0] - torch.from_numpy(target)) ** 2)
            loss.backward()
            assert sched.adjoint_steps == T
            grads[precision] = ({k: ts[k].grad.numpy().copy() for k in VEL}, float(rho.grad), float(loss))

    # central differences of the plain FP64 forward
    with fs.Solver(n, dx, **params(fs.FS_PRECISION_FP64, 1e-12)) as s:
        def loss_fd(st, rho_w):
            s.set_params(rho_neg=rho_w)
            s.upload("pressure", np.zeros((n, n, n)))
            for k in KEYS:
                s.upload(k, st[k])
            for _ in range(T):
                s.step(dt)
            return float(np.sum((s.download("phi") - target) ** 2))

        h = 1e-6
        fds = []
        ads = {fs.FS_PRECISION_FP32_REFINE: [], fs.FS_PRECISION_FP64: []}
        for d in range(1, 17):
            r = np.random.default_rng(d)
            dX = zero_walls({"phi": X["phi"], "u": r.normal(size=X["u"].shape), "v": r.normal(size=X["v"].shape),
                             "w": r.normal(size=X["w"].shape)})
            norm = np.sqrt(sum(np.sum(dX[k] ** 2) for k in VEL))
            dX = {k: dX[k] / norm for k in VEL}
            plus = {k: X[k] + h * dX[k] if k in dX else X[k] for k in KEYS}
            minus = {k: X[k] - h * dX[k] if k in dX else X[k] for k in KEYS}
            fd = (loss_fd(plus, 1000.0) - loss_fd(minus, 1000.0)) / (2 * h)
            fds.append(fd)
            for prec, (g, _, _) in grads.items():
                ads[prec].append(sum(float(np.sum(g[k] * dX[k])) for k in VEL))
        hr = 0.5
        fd_rho = (loss_fd(X, 1000.0 + hr) - loss_fd(X, 1000.0 - hr)) / (2 * hr)
    # each direction's error relative to its own derivative, floored at a
    # tenth of the largest directional derivative: a direction along which
    # the loss hardly changes is compared on the gradient's scale, not on its
    # own near-zero value (where the finite difference is mostly noise)
    fds = np.array(fds)
    floor = 0.1 * np.abs(fds).max()
    errs = {}
    for prec, name in ((fs.FS_PRECISION_FP32_REFINE, "FP32"), (fs.FS_PRECISION_FP64, "FP64")):
        a = np.array(ads[prec])
        errs[prec] = np.abs(a - fds) / np.maximum(np.abs(fds), floor)
        print(f"96^3 x 32 dam break, {name} adjoint: loss {grads[prec][2]:.6e}, max relative FD error over 16 "
              f"directions {errs[prec].max():.2e} (median {np.median(errs[prec]):.2e}), density ratio "
              f"{grads[prec][1]:.6e} vs FD {fd_rho:.6e}")
        for d in range(16):
            print(f"  direction {d + 1:2d}: FD {fds[d]:+.9e} adjoint {a[d]:+.9e} error {errs[prec][d]:.2e}")
    assert max(errs[fs.FS_PRECISION_FP64]) < 1e-4
    assert max(errs[fs.FS_PRECISION_FP32_REFINE]) < 1e-2
    assert rel(grads[fs.FS_PRECISION_FP64][1], fd_rho) < 1e-3
    assert rel(grads[fs.FS_PRECISION_FP32_REFINE][1], fd_rho) < 1e-2


@pytest.mark.parametrize("op", ["step", "projection", "viscosity"])
def test_fp32_adjoint_transpose(op):
    """Dot-product test in the FP32 + FP64 refinement context: <Ybar, J dX>
    by central differences of the context's own FP32 forward (h = 1e-3, so
    that FP32 rounding of the outputs, about 1e-7, stays near 1e-4 of the
    difference) against <Jt Ybar, dX> from its adjoint.  A transposition
error shows as an O(1) mismatch; the 1e-2 bound leaves room for the
rounding and the WENO weights' curvature at this step size."""
    from test_adjoint import rand_like, rel, scene, transpose_check
    from test_adjoint import zero_walls as zw
    n = 10
    X = zw(scene(n, 7, vel_scale=0.2))
    rng = np.random.default_rng(40)
    dX = zw(rand_like(X, rng, KEYS))
    dX["phi"] = dX["phi"] * 0.01
    Ybar = rand_like(X, rng, KEYS)
    dt = 0.3 / n
    rho, drho = (1.0, 1000.0), (0.2, 50.0)
    p = dict(rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, precision=fs.FS_PRECISION_FP32_REFINE,
             tolerance=1e-12, stop=fs.FS_STOP_RELATIVE, max_iteration=100000, viscosity=1,
             viscosity_tolerance=1e-12, viscosity_max_iteration=100000, order=3)
    if op == "viscosity":
        p.update(mu_neg=2e-2, mu_pos=5e-2)  # large enough that the coefficients matter
    fwd, adj, outs = {"step": (lambda s: s.step(dt), lambda s: s.step_adjoint(dt), KEYS),
                      "projection": (lambda s: s.project(dt), lambda s: s.project_adjoint(dt), VEL),
                      "viscosity": (lambda s: s.viscosity(dt), lambda s: s.viscosity_adjoint(dt), VEL)}[op]
    with fs.Solver(n, 1.0 / n, **p) as s:
        lhs, rhs = transpose_check(s, fwd, adj, X, dX, Ybar, outs, KEYS, 1e-3, rho, drho)
    print(f"FP32 context, {op}: <Ybar, J dX> {lhs:.9e}, <Jt Ybar, dX> {rhs:.9e}, relative {rel(lhs, rhs):.2e}")
    assert rel(lhs, rhs) < 1e-2, (lhs, rhs)
