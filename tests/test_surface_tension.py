"""Surface tension on the GPU (through the C ABI) against the oracle and the
reference's own outputs: curvature (LEVELSET_3D::ComputeCurvatures), the
ghost-fluid jump terms of the pressure right-hand side and velocity update
(POISSON_SOLVER_3D.h:1216-1328, PROJECTION_3D.h:1181), the CFL term, and a
whole step."""
import os

import numpy as np
import pytest

import fluid_simulator_backup_b200 as fs
from oracle import fs_oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
pytestmark = pytest.mark.gpu
SIGMA = 0.0728


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def sphere(n, c, r, noise=0.0, seed=0):
    x = (np.arange(n) + 0.5) / n
    phi = np.sqrt((x[None, None, :] - c[0]) ** 2 + (x[None, :, None] - c[1]) ** 2 + (x[:, None, None] - c[2]) ** 2) - r
    return phi + noise * np.random.default_rng(seed).normal(size=phi.shape)


def make(n, precision=fs.FS_PRECISION_FP64, **kw):
    return fs.Solver(n, 1.0 / n, precision=precision, **kw)


def upload_all(s, phi, u, v, w):
    for k, a in zip(("phi", "u", "v", "w"), (phi, u, v, w)):
        s.upload(k, a)


@pytest.mark.parametrize("typo", [False, True])
def test_curvature_matches_oracle(typo):
    n = 18
    phi = sphere(n, (0.5, 0.45, 0.55), 0.3, noise=2e-3, seed=1)
    with make(n, flags=fs.FS_FLAG_CURVATURE_TYPO if typo else 0) as s:
        s.upload("phi", phi)
        kappa, kmax = s.curvature()
    ref, ref_max = O.curvature(phi, 1.0 / n, typo=typo)
    assert rel_err(kappa, ref) < 1e-12
    assert abs(kmax - ref_max) <= 1e-12 * ref_max


def test_projection_with_surface_tension_matches_reference_golden():
    """The reference's own projection with sigma = 0.0728 (faithful mode and the
    reference's curvature slips): right-hand side with jump terms, PCG, and
    the velocity update with the interface jump."""
    g = dict(np.load(os.path.join(GOLD, "projection_tension.npz")))
    n = int(g["n"])
    with make(n, rho_neg=float(g["rho_neg"]), rho_pos=float(g["rho_pos"]), tolerance=float(g["tol"]),
              stop=fs.FS_STOP_ABSOLUTE, max_iteration=100000, surface_tension=float(g["sigma"]),
              flags=fs.FS_FLAG_FAITHFUL_PROJECTION | fs.FS_FLAG_CURVATURE_TYPO) as s:
        upload_all(s, g["phi"], g["u"], g["v"], g["w"])
        s.upload("pressure", np.zeros((n, n, n)))
        rep = s.project(float(g["dt"]))
        p = s.download("pressure")
        vel = [s.download(k) for k in "uvw"]
    assert abs(rep["iterations"] - int(g["iterations"])) <= 2
    assert rel_err(p, g["out_p"]) < 1e-7
    for k, a in zip("uvw", vel):
        assert rel_err(a, g["out_" + k]) < 1e-7


@pytest.mark.parametrize("precision,tol", [(fs.FS_PRECISION_FP64, 1e-9), (fs.FS_PRECISION_FP32_REFINE, 1e-6)])
def test_corrected_projection_with_surface_tension_matches_oracle(precision, tol):
    n = 20
    phi = sphere(n, (0.5, 0.4, 0.5), 0.25, noise=1e-3, seed=2)
    rng = np.random.default_rng(3)
    u = rng.normal(size=(n, n, n + 1)) * 0.2
    v = rng.normal(size=(n, n + 1, n)) * 0.2
    w = rng.normal(size=(n + 1, n, n)) * 0.2
    u[:, :, 0] = u[:, :, -1] = 0; v[:, 0, :] = v[:, -1, :] = 0; w[0] = w[-1] = 0
    dt = 2e-3
    with make(n, precision, rho_neg=1.0, rho_pos=1000.0, tolerance=1e-12, stop=fs.FS_STOP_RELATIVE,
              max_iteration=100000, surface_tension=SIGMA) as s:
        upload_all(s, phi, u, v, w)
        s.project(dt)
        got = [s.download(k) for k in "uvw"]
    ref = O.projection(phi, u, v, w, 1.0 / n, dt, 1.0, 1000.0, 1e-13, 100000, mode="corrected", criterion="rel",
                       sigma=SIGMA)
    for a, b in zip(got, ref[:3]):
        assert rel_err(a, b) < tol


def test_cfl_includes_the_surface_tension_term():
    n = 16
    phi = sphere(n, (0.5, 0.5, 0.5), 0.2, noise=1e-3, seed=4)
    rng = np.random.default_rng(5)
    u = rng.normal(size=(n, n, n + 1)) * 0.01
    v = rng.normal(size=(n, n + 1, n)) * 0.01
    w = rng.normal(size=(n + 1, n, n)) * 0.01
    with make(n, rho_neg=1.0, rho_pos=1000.0, viscosity=1, cfl=1.0, surface_tension=SIGMA) as s:
        upload_all(s, phi, u, v, w)
        dt = s.cfl_dt()
    _, kmax = O.curvature(phi, 1.0 / n)
    s_f = np.sqrt((SIGMA * kmax) / (min(1.0, 1000.0) * (1.0 / n) ** 2))
    ref = O.cfl_dt(u, v, w, 1.0 / n, -9.8, 0.0, s_f)
    assert abs(dt - ref) <= 1e-13 * ref
    assert dt < O.cfl_dt(u, v, w, 1.0 / n, -9.8, 0.0, 0.0)


def test_whole_step_with_surface_tension_matches_oracle():
    n = 16
    dx = 1.0 / n
    phi = sphere(n, (0.5, 0.35, 0.5), 0.2, noise=1e-3, seed=6)
    u = np.zeros((n, n, n + 1)); v = np.zeros((n, n + 1, n)); w = np.zeros((n + 1, n, n))
    P = dict(rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, gravity=(0.0, -9.8, 0.0), eps=1e-6,
             reinit_iterations=10, reinit_scaling=5, tol=1e-12, max_iter=20000, viscosity=True, visc_tol=1e-12,
             sigma=SIGMA)
    with make(n, rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, tolerance=1e-12, stop=fs.FS_STOP_RELATIVE,
              viscosity_tolerance=1e-12, surface_tension=SIGMA) as s:
        upload_all(s, phi, u, v, w)
        dt = s.cfl_dt()
        s.step(dt)
        got = [s.download(k) for k in ("phi", "u", "v", "w")]
    ref = O.step(phi, u, v, w, dx, dt, P)
    for a, b in zip(got, ref[:4]):
        assert rel_err(a, b) < 1e-8
