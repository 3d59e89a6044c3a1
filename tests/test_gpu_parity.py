"""Parity of the CUDA path (through the C ABI) with the oracle and with the
reference's own outputs (golden fixtures).

Tolerances: FP64 kernels agree with the FP64 oracle to 1e-10 relative (the
kernels use fused multiply-adds and one-division WENO weights, the oracle the
reference's exact expression order); FP32 storage/arithmetic to 2e-5 relative
for single operators.  Iterative solves are compared at their solver
tolerance."""
import os

import numpy as np
import pytest

import fluid_simulator_backup_b200 as fs
from oracle import fs_oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
pytestmark = pytest.mark.gpu


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def random_state(n, seed, scale=0.3):
    rng = np.random.default_rng(seed)
    nx, ny, nz = n
    phi = rng.normal(size=(nz, ny, nx)) * 0.1
    u = rng.normal(size=(nz, ny, nx + 1)) * scale
    v = rng.normal(size=(nz, ny + 1, nx)) * scale
    w = rng.normal(size=(nz + 1, ny, nx)) * scale
    return phi, u, v, w


def sphere(n, c, r):
    x = (np.arange(n) + 0.5) / n
    return np.sqrt((x[None, None, :] - c[0]) ** 2 + (x[None, :, None] - c[1]) ** 2 + (x[:, None, None] - c[2]) ** 2) - r


def make(n, precision=fs.FS_PRECISION_FP64, **kw):
    if isinstance(n, int):
        n = (n, n, n)
    return fs.Solver(n, 1.0 / n[0], precision=precision, **kw)


def upload_all(s, phi, u, v, w):
    for k, a in zip(("phi", "u", "v", "w"), (phi, u, v, w)):
        s.upload(k, a)


@pytest.mark.parametrize("precision,tol", [(fs.FS_PRECISION_FP64, 1e-10), (fs.FS_PRECISION_FP32_REFINE, 2e-5)])
def test_weno5_levelset_matches_oracle(precision, tol):
    n = (20, 17, 13)
    phi, u, v, w = random_state(n, 1)
    with make(n, precision) as s:
        upload_all(s, phi, u, v, w)
        s.advect_levelset(2e-3)
        got = s.download("phi")
    ref = O.weno5_levelset(phi, u, v, w, 1.0 / n[0], 2e-3, 1e-6)
    assert rel_err(got, ref) < tol


@pytest.mark.parametrize("precision,tol", [(fs.FS_PRECISION_FP64, 1e-10), (fs.FS_PRECISION_FP32_REFINE, 2e-5)])
def test_weno5_velocity_matches_oracle(precision, tol):
    n = (16, 18, 14)
    phi, u, v, w = random_state(n, 2)
    with make(n, precision) as s:
        upload_all(s, phi, u, v, w)
        s.advect_velocity(2e-3)
        got = [s.download(k) for k in "uvw"]
    ref = O.weno5_velocity(u, v, w, 1.0 / n[0], 2e-3, 1e-6)
    for g, r in zip(got, ref):
        assert rel_err(g, r) < tol


@pytest.mark.parametrize("typo", [False, True])
def test_reinitialization_matches_oracle(typo):
    n = 16
    phi = np.random.default_rng(3).normal(size=(n, n, n)) * 0.1
    flags = fs.FS_FLAG_REINIT_TYPO if typo else 0
    with make(n, flags=flags) as s:
        s.upload("phi", phi)
        s.reinitialize()
        got = s.download("phi")
    ref = O.reinitialization_block(phi, 1.0 / n, 10, 5, 1e-6, typo=typo)
    assert rel_err(got, ref) < 1e-9


def test_golden_weno_and_reinit_through_cuda():
    g = load("weno5_levelset")
    n = int(g["n"])
    with make(n) as s:
        upload_all(s, g["phi"], g["u"], g["v"], g["w"])
        s.advect_levelset(float(g["dt"]))
        assert rel_err(s.download("phi"), g["out"]) < 1e-10
    g = load("weno5_velocity")
    n = int(g["n"])
    with make(n) as s:
        upload_all(s, np.zeros((n, n, n)), g["u"], g["v"], g["w"])
        s.advect_velocity(float(g["dt"]))
        for k in "uvw":
            assert rel_err(s.download(k), g["out_" + k]) < 1e-10
    g = load("reinit")
    n = int(g["n"])
    with make(n, flags=fs.FS_FLAG_REINIT_TYPO) as s:
        s.upload("phi", g["phi"])
        s.reinitialize()
        assert rel_err(s.download("phi"), g["out"]) < 1e-9


@pytest.mark.parametrize("name", ["projection_drop", "projection_bubble"])
def test_golden_projection_faithful_through_cuda(name):
    """The reference's PROJECTION_3D::Solve output (w-only update, absolute
    r.z < tol^2 stop) reproduced by the CUDA path in faithful mode."""
    g = load(name)
    n = int(g["n"])
    with make(n, rho_neg=float(g["rho_neg"]), rho_pos=float(g["rho_pos"]), stop=fs.FS_STOP_ABSOLUTE,
              tolerance=float(g["tol"]), max_iteration=100000, flags=fs.FS_FLAG_FAITHFUL_PROJECTION) as s:
        upload_all(s, g["phi"], g["u"], g["v"], g["w"])
        rep = s.project(float(g["dt"]))
        p = s.download("pressure")
        vel = [s.download(k) for k in "uvw"]
        div = s.download("divergence")
    assert rel_err(div, g["div"]) < 1e-12
    assert abs(rep["iterations"] - int(g["iterations"])) <= 2
    assert rel_err(p, g["out_p"]) < 1e-7
    for k, a in zip("uvw", vel):
        assert rel_err(a, g["out_" + k]) < 1e-7


def test_golden_linear_solver_plugin_csr():
    """LINEAR_SOLVER plugin: the reference's own CSR system and PCG solution."""
    g = load("projection_bubble")
    x, it, res, status = fs.pcg_csr(g["csr_vals"], g["csr_cols"], g["csr_rowptr"], g["b"], np.zeros_like(g["b"]),
                                    float(g["tol"]), 100000, fs.FS_STOP_ABSOLUTE)
    assert status == fs.FS_OK
    assert abs(it - int(g["iterations"])) <= 2
    assert rel_err(x, g["x"]) < 1e-7


@pytest.mark.parametrize("precision", [fs.FS_PRECISION_FP64, fs.FS_PRECISION_FP32_REFINE])
def test_projection_corrected_matches_oracle(precision):
    n = 24
    rng = np.random.default_rng(5)
    phi = sphere(n, (0.5, 0.4, 0.5), 0.25)
    _, u, v, w = random_state((n, n, n), 6)
    u, v, w = O.zero_walls(u, v, w)  # no net flux through the walls: the projected field can be divergence free
    dx, dt = 1.0 / n, 1e-3
    with make(n, precision, rho_neg=1.0, rho_pos=1000.0, tolerance=1e-9, max_iteration=20000) as s:
        upload_all(s, phi, u, v, w)
        rep = s.project(dt)
        p = s.download("pressure")
        vel = [s.download(k) for k in "uvw"]
    ru, rv, rw, rp, info = O.projection(phi, u, v, w, dx, dt, 1.0, 1000.0, 1e-12, 20000, mode="corrected",
                                        criterion="rel")
    assert rep["rel_residual"] < 1e-9
    tol = 1e-6 if precision == fs.FS_PRECISION_FP64 else 2e-5
    # the corrected system is the singular Neumann system: pressure up to a constant
    assert rel_err(p - p.mean(), rp - rp.mean()) < tol
    for a, b in zip(vel, (ru, rv, rw)):
        assert rel_err(a, b) < tol
    # the corrected update is the gradient the pressure matrix was built from,
    # so the velocity's divergence is dt times the solve's residual: relative
    # to the input's divergence it is below the solve tolerance, the
    # interface included, up to the rounding of the stored velocities (FP32:
    # eps32 |u| / dx per cell)
    div_in = np.linalg.norm(O.divergence(u, v, w, dx, 1.0))
    vmax = max(np.abs(a).max() for a in vel)
    floor = 0.0 if precision == fs.FS_PRECISION_FP64 else 4 * 6e-8 * vmax / dx * np.sqrt(n ** 3)
    assert rep["div_l2"] <= 2e-9 * div_in + 1e-12 + floor, (rep["div_l2"], div_in, floor)
    assert rel_err(np.linalg.norm(O.divergence(*vel, dx, 1.0)), rep["div_l2"]) < 1e-6 or rep["div_l2"] < 1e-10


def test_faithful_projection_keeps_the_reference_interface_residual():
    """FS_FLAG_FAITHFUL_PROJECTION reproduces the reference's update (w only,
    smeared interface density), which is not the matrix's gradient: a
    divergence residual stays, as in the oracle's faithful mode."""
    n = 16
    phi = sphere(n, (0.5, 0.4, 0.5), 0.25)
    _, u, v, w = random_state((n, n, n), 6)
    dx, dt = 1.0 / n, 1e-3
    with make(n, rho_neg=1.0, rho_pos=1000.0, tolerance=1e-12, max_iteration=20000,
              flags=fs.FS_FLAG_FAITHFUL_PROJECTION) as s:
        upload_all(s, phi, u, v, w)
        rep = s.project(dt)
        vel = [s.download(k) for k in "uvw"]
    ru, rv, rw, rp, info = O.projection(phi, u, v, w, dx, dt, 1.0, 1000.0, 1e-13, 20000, mode="faithful",
                                        criterion="rel")
    for a, b in zip(vel, (ru, rv, rw)):
        assert rel_err(a, b) < 1e-8
    div_ref = np.linalg.norm(O.divergence(ru, rv, rw, dx, 1.0))
    assert div_ref > 1e-3 * np.linalg.norm(O.divergence(u, v, w, dx, 1.0))
    assert rel_err(rep["div_l2"], div_ref) < 1e-6


def test_bf16_jacobi_preconditioner():
    """The FP32 pressure solve preconditioned by 1/diag rounded to bf16
    against the exact FP32 diagonal: any fixed SPD diagonal is a valid
    Jacobi preconditioner, both reach the same FP64 true residual, so the
    pressures agree to the solve tolerance and the iteration counts stay
    close."""
    n = 48
    phi = sphere(n, (0.5, 0.4, 0.5), 0.2)
    _, u, v, w = random_state((n, n, n), 9)
    dt = 1e-3
    out = {}
    for mode in (fs.FS_PRECOND_JACOBI, fs.FS_PRECOND_JACOBI_BF16):
        with make(n, fs.FS_PRECISION_FP32_REFINE, rho_neg=1.0, rho_pos=1000.0, tolerance=1e-10,
                  max_iteration=20000, pressure_preconditioner=mode) as s:
            upload_all(s, phi, u, v, w)
            rep = s.project(dt)
            out[mode] = (rep, s.download("pressure"))
    (r0, p0), (r1, p1) = out[fs.FS_PRECOND_JACOBI], out[fs.FS_PRECOND_JACOBI_BF16]
    assert r0["rel_residual"] < 1e-10 and r1["rel_residual"] < 1e-10
    assert abs(r1["iterations"] - r0["iterations"]) <= 0.1 * r0["iterations"] + 16
    p0 = p0 - p0.mean()
    p1 = p1 - p1.mean()
    assert rel_err(p1, p0) < 1e-7


def test_viscosity_matches_oracle():
    n = 16
    phi = sphere(n, (0.5, 0.5, 0.5), 0.3)
    _, u, v, w = random_state((n, n, n), 7)
    u, v, w = O.zero_walls(u, v, w)
    dx, dt = 1.0 / n, 5e-3
    with make(n, rho_neg=1.0, rho_pos=1000.0, mu_neg=0.05, mu_pos=0.2, viscosity_tolerance=1e-12) as s:
        upload_all(s, phi, u, v, w)
        s.viscosity(dt)
        got = [s.download(k) for k in "uvw"]
    ref, _ = O.viscosity_semi_implicit(phi, u, v, w, dx, dt, 1.0, 1000.0, 0.05, 0.2, 1e-13, 10000)
    for a, b in zip(got, ref):
        assert rel_err(a, b) < 1e-8


def test_cfl_matches_reference_formula():
    g = load("cfl")
    n = int(g["n"])
    with make(n, viscosity=0, cfl=1.0, mu_neg=1e-3, mu_pos=1.8e-5, rho_neg=1000.0, rho_pos=1.0) as s:
        upload_all(s, np.zeros((n, n, n)), g["u"], g["v"], g["w"])
        assert abs(s.cfl_dt() - float(g["out"])) < 1e-14 * float(g["out"])


@pytest.mark.parametrize("order", [1, 3])
@pytest.mark.parametrize("precision,tol", [(fs.FS_PRECISION_FP64, 1e-8), (fs.FS_PRECISION_FP32_REFINE, 5e-4)])
def test_whole_step_matches_oracle(precision, tol, order):
    """Two full timesteps (with semi-implicit viscosity) against the oracle's
    corrected step, both pressure solves stopped at a 1e-12 relative
    residual; fields compared relative to their maximum: 1e-8 in FP64, 5e-4
    with FP32 storage."""
    n = 16
    dx = 1.0 / n
    phi = sphere(n, (0.5, 0.35, 0.5), 0.2)
    u = np.zeros((n, n, n + 1)); v = np.zeros((n, n + 1, n)); w = np.zeros((n + 1, n, n))
    P = dict(rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, gravity=(0.0, -9.8, 0.0), eps=1e-6,
             reinit_iterations=10, reinit_scaling=5, tol=1e-12, max_iter=20000, viscosity=True, visc_tol=1e-12)
    # the FP64 defect residual of the FP32 path floors near 1e-11 here
    ptol = 1e-12 if precision == fs.FS_PRECISION_FP64 else 1e-10
    with make(n, precision, rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, tolerance=ptol,
              viscosity_tolerance=1e-12, order=order) as s:
        upload_all(s, phi, u, v, w)
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


def test_error_paths_leave_context_usable():
    n = 12
    phi = sphere(n, (0.5, 0.5, 0.5), 0.3)
    _, u, v, w = random_state((n, n, n), 9)
    with make(n, rho_neg=1.0, rho_pos=1000.0) as s:
        upload_all(s, phi, u, v, w)
        # iteration cap -> NOT_CONVERGED, context still usable
        s.set_params(max_iteration=1)
        rep = s.project(1e-3, allow_not_converged=True)
        assert rep["status"] == fs.FS_NOT_CONVERGED
        s.set_params(max_iteration=20000)
        upload_all(s, phi, u, v, w)
        assert s.project(1e-3)["status"] == fs.FS_OK
        # non-finite input -> NONFINITE
        bad = u.copy()
        bad[3, 4, 5] = np.nan
        s.upload("u", bad)
        with pytest.raises(fs.FsError) as e:
            s.project(1e-3)
        assert e.value.status == fs.FS_NONFINITE
        upload_all(s, phi, u, v, w)
        assert s.project(1e-3)["status"] == fs.FS_OK
        with pytest.raises(ValueError):
            s.upload("u", np.zeros((3, 3, 3)))
        with pytest.raises(fs.FsError):
            s.step(-1.0)
