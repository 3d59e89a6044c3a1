"""The red-black reduced pressure solve of the FP32 + FP64 refinement path
(FS_PRECOND_RED_BLACK): the reference's Jacobi-PCG (PCG_METHOD.cpp:4-126) in
red-black order, red cells eliminated exactly, CG on the black Schur
complement.  Checked through the C ABI against the FP64 oracle's projection
and the full-system Jacobi solve: same pressure and velocities to the solve
tolerance, about half the iterations, divergence free to the tolerance."""
import numpy as np
import pytest

import fluid_simulator_backup_b200 as fs
from oracle import fs_oracle as O

pytestmark = pytest.mark.gpu


def sphere(n, c, r):
    nx, ny, nz = n
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / nx
    z = (np.arange(nz) + 0.5) / nx
    return np.sqrt((x[None, None, :] - c[0]) ** 2 + (y[None, :, None] - c[1]) ** 2 + (z[:, None, None] - c[2]) ** 2) - r


def velocities(n, seed, scale=0.3):
    nx, ny, nz = n
    rng = np.random.default_rng(seed)
    u = rng.normal(size=(nz, ny, nx + 1)) * scale
    v = rng.normal(size=(nz, ny + 1, nx)) * scale
    w = rng.normal(size=(nz + 1, ny, nx)) * scale
    return O.zero_walls(u, v, w)


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def solver(n, precond, precision=fs.FS_PRECISION_FP32_REFINE, **kw):
    return fs.Solver(n, 1.0 / n[0], precision=precision, rho_neg=1.0, rho_pos=1000.0, max_iteration=40000,
                     pressure_preconditioner=precond, **kw)


@pytest.mark.parametrize("precond", ["ic0", "jacobi"])
@pytest.mark.parametrize("n", [(24, 24, 24), (17, 14, 15), (32, 20, 9)])
def test_red_black_projection_matches_oracle(n, precond):
    """Even and odd extents (odd nx leaves slots of the packed half layout
    without a cell): pressure and corrected velocities equal the oracle's
    FP64 projection to the tolerance, and the corrected velocity is divergence
    free to it."""
    nx = n[0]
    dx, dt = 1.0 / nx, 1e-3
    phi = sphere(n, (0.5, 0.3, 0.25), 0.17)
    u, v, w = velocities(n, 3)
    pc = fs.FS_PRECOND_RED_BLACK if precond == "ic0" else fs.FS_PRECOND_RED_BLACK_JACOBI
    with solver(n, pc, tolerance=1e-10) as s:
        for k, a in zip(("phi", "u", "v", "w"), (phi, u, v, w)):
            s.upload(k, a)
        rep = s.project(dt)
        p = s.download("pressure")
        vel = [s.download(k) for k in "uvw"]
    ru, rv, rw, rp, info = O.projection(phi, u, v, w, dx, dt, 1.0, 1000.0, 1e-13, 40000, mode="corrected",
                                        criterion="rel")
    assert rep["rel_residual"] <= 1e-10
    p = p - p.mean()
    rp = rp - rp.mean()
    assert rel_err(p, rp) < 2e-6
    for a, b in zip(vel, (ru, rv, rw)):
        assert rel_err(a, b) < 2e-5
    div_in = np.linalg.norm(O.divergence(u, v, w, dx, 1.0))
    vmax = max(np.abs(a).max() for a in vel)
    floor = 4 * 6e-8 * vmax / dx * np.sqrt(np.prod(n))
    assert rep["div_l2"] <= 2e-10 * div_in + floor


def test_red_black_needs_about_half_the_jacobi_iterations():
    """For a two-coloured operator the Schur complement's Jacobi spectrum is
    {1 - l^2} against {1 +- l}: CG needs about half the iterations of the
    full Jacobi-PCG at the same tolerance, and both reach the same pressure.
    The IC(0) pivots diag(S) are at least as good a scaling of S as the
    black cells' own diagonal."""
    n = (48, 48, 48)
    phi = sphere(n, (0.5, 0.25, 0.5), 0.15)
    u, v, w = velocities(n, 4, 0.1)
    out = {}
    for precond in (fs.FS_PRECOND_JACOBI_BF16, fs.FS_PRECOND_RED_BLACK, fs.FS_PRECOND_RED_BLACK_JACOBI):
        with solver(n, precond, tolerance=1e-8) as s:
            for k, a in zip(("phi", "u", "v", "w"), (phi, u, v, w)):
                s.upload(k, a)
            rep = s.project(2e-3)
            out[precond] = (rep, s.download("pressure"))
    (rj, pj), (rr, pr), (rb, pb) = (out[fs.FS_PRECOND_JACOBI_BF16], out[fs.FS_PRECOND_RED_BLACK],
                                    out[fs.FS_PRECOND_RED_BLACK_JACOBI])
    print(f"48^3 projection to 1e-8: Jacobi {rj['iterations']} iterations, red-black IC(0) {rr['iterations']}, "
          f"red-black with the black diagonal {rb['iterations']}")
    for r in (rj, rr, rb):
        assert r["rel_residual"] <= 1e-8
    assert rr["iterations"] < 0.65 * rj["iterations"], (rr["iterations"], rj["iterations"])
    assert rb["iterations"] < 0.65 * rj["iterations"], (rb["iterations"], rj["iterations"])
    assert rr["iterations"] <= 1.05 * rb["iterations"], (rr["iterations"], rb["iterations"])
    assert rel_err(pr - pr.mean(), pj - pj.mean()) < 1e-6
    assert rel_err(pb - pb.mean(), pj - pj.mean()) < 1e-6


@pytest.mark.parametrize("order", [1, 3])
def test_red_black_whole_step_matches_oracle(order):
    """Two whole timesteps (advection, gravity, semi-implicit viscosity, the
    projections, reinitialisation) with the red-black pressure solve against
    the oracle's FP64 step, compared as the full-system FP32 path is: fields
    relative to their maximum within 5e-4 (FP32 storage)."""
    n = 16
    dx = 1.0 / n
    phi = sphere((n, n, n), (0.5, 0.35, 0.5), 0.2)
    u = np.zeros((n, n, n + 1)); v = np.zeros((n, n + 1, n)); w = np.zeros((n + 1, n, n))
    P = dict(rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, gravity=(0.0, -9.8, 0.0), eps=1e-6,
             reinit_iterations=10, reinit_scaling=5, tol=1e-12, max_iter=20000, viscosity=True, visc_tol=1e-12)
    tol = 5e-4
    with solver((n, n, n), fs.FS_PRECOND_RED_BLACK, mu_neg=1.8e-5, mu_pos=1e-3, tolerance=1e-10,
                viscosity_tolerance=1e-12, order=order) as s:
        for k, a in zip(("phi", "u", "v", "w"), (phi, u, v, w)):
            s.upload(k, a)
        dt = s.cfl_dt()
        states = []
        p0 = None
        ph, uu, vv, ww = phi, u, v, w
        for _ in range(2):
            rep = s.step(dt)
            assert rep["projections"] == order
            ph, uu, vv, ww, p0, info = O.step(ph, uu, vv, ww, dx, dt, P, p0, order=order)
            states.append(([s.download(k) for k in ("phi", "u", "v", "w")], (ph, uu, vv, ww)))
    for got, ref in states:
        assert rel_err(got[0], ref[0]) < max(tol / 10, 1e-6)
        for a, b in zip(got[1:], ref[1:]):
            assert np.abs(a - b).max() < tol * max(np.abs(b).max(), 1e-3)
