"""Oil/water vertical pipe mode through the CUDA path against the reference's
own outputs (fixtures pipe_*, made by tests/golden/make_golden.py from the
headless reference build) and against the oracle.

The pipe mode's level-set advection, reinitialisation, ENO3 velocity
advection, dimensionless body force, projection and CFL time step run on the
GPU, and so does the whole step without viscosity (the reference's step with
is_sourcing_active = false); the pipe's viscosity is not built, and that
entry point (with fs_step when viscosity != 0) returns FS_NOT_SUPPORTED in
this mode."""
import os

import numpy as np
import pytest

import fluid_simulator_backup_b200 as fs
from oracle import fs_oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def solver(g, precision=fs.FS_PRECISION_FP64, flags=fs.FS_FLAG_REINIT_TYPO, **kw):
    n = tuple(int(x) for x in g["n"])
    dx = (float(g["hi"][0]) - float(g["lo"][0])) / (n[0] - 1)
    # the projection's dimensionless densities: 1 in the oil (phi <= 0),
    # water_density/oil_density in the water (PROJECTION_3D.h:642-669)
    water = float(g["water_density"]) if "water_density" in g else 0.995
    args = dict(precision=precision, pipe=1, pipe_radius=float(g["a"]), grid_min=tuple(g["lo"]),
                grid_max=tuple(g["hi"]), pipe_R1=float(g["R1"]), pipe_V0=float(g["V0"]), pipe_f=float(g["f"]),
                pipe_eta=float(g["eta"]), pipe_oil_density=float(g["oil_density"]), pipe_We=float(g["We"]),
                rho_neg=1.0, rho_pos=water / float(g["oil_density"]),
                gravity=(0.0, float(g["gravity_y"]), 0.0), weno_epsilon=float(g["epsilon"]),
                reinit_iterations=int(g["reinit_iterations"]), reinit_scaling=int(g["reinit_scaling"]),
                flags=flags, viscosity=0, velocity_scheme=fs.FS_VELOCITY_ENO3)
    args.update(kw)
    return fs.Solver(n, dx, **args)


def upload(s, g, keys=("phi", "u", "v", "w")):
    for k in keys:
        s.upload(k, g[k])


@pytest.mark.parametrize("precision,tol", [(fs.FS_PRECISION_FP64, 1e-12), (fs.FS_PRECISION_FP32_REFINE, 2e-5)])
def test_pipe_levelset_advection_matches_reference(precision, tol):
    g = load("pipe_levelset")
    with solver(g, precision) as s:
        upload(s, g)
        s.advect_levelset(float(g["dt"]))
        phi = s.download("phi")
        scale = np.abs(g["phi"]).max()
        assert np.abs(phi - g["out_phi"]).max() <= tol * scale
        b = g["boundary"]
        # cells outside the pipe keep their value (exactly: they are copied)
        assert np.abs(phi[b > 0] - g["phi"][b > 0]).max() <= (0.0 if precision == fs.FS_PRECISION_FP64 else 1e-6)
        for k in "uvw":
            out = s.download(k)
            assert np.abs(out - g["out_" + k]).max() <= tol * max(np.abs(g[k]).max(), 1.0), k


@pytest.mark.parametrize("precision,tol", [(fs.FS_PRECISION_FP64, 1e-9), (fs.FS_PRECISION_FP32_REFINE, 2e-5)])
def test_pipe_reinitialization_matches_reference(precision, tol):
    g = load("pipe_reinit")
    with solver(g, precision) as s:
        upload(s, g, ("phi",))
        s.reinitialize()
        out = s.download("phi")
        assert np.abs(out - g["out_phi"]).max() <= tol * np.abs(g["phi"]).max()
    # the corrected tree (no typo leaves) against the oracle
    grids = O.pipe_grids(tuple(int(x) for x in g["n"]), tuple(g["lo"]), tuple(g["hi"]))
    ref = O.pipe_reinitialization(g["phi"], grids, int(g["reinit_iterations"]), int(g["reinit_scaling"]),
                                  float(g["epsilon"]), typo=False)
    with solver(g, fs.FS_PRECISION_FP64, flags=0) as s:
        upload(s, g, ("phi",))
        s.reinitialize()
        assert np.abs(s.download("phi") - ref).max() <= 1e-9 * np.abs(g["phi"]).max()


@pytest.mark.parametrize("precision,tol", [(fs.FS_PRECISION_FP64, 1e-12), (fs.FS_PRECISION_FP32_REFINE, 2e-6)])
def test_pipe_forcing_matches_reference(precision, tol):
    g = load("pipe_forcing")
    with solver(g, precision) as s:
        upload(s, g)
        s.apply_gravity(float(g["dt"]))
        step = np.abs(g["out_v"] - g["v"]).max()
        assert step > 0
        assert np.abs(s.download("v") - g["out_v"]).max() <= tol * max(np.abs(g["v"]).max(), 1.0)
        # u and w are untouched, the fixed centre line keeps its value
        for k in "uw":
            assert np.abs(s.download(k) - g[k]).max() <= (0.0 if precision == fs.FS_PRECISION_FP64 else 1e-6)
        v = s.download("v")
        fixed = g["fixed_v"]
        assert np.abs(v[fixed] - g["v"][fixed]).max() <= (0.0 if precision == fs.FS_PRECISION_FP64 else 1e-6)


@pytest.mark.parametrize("precision,tol", [(fs.FS_PRECISION_FP64, 1e-12), (fs.FS_PRECISION_FP32_REFINE, 2e-5)])
def test_pipe_velocity_advection_matches_reference(precision, tol):
    g = load("pipe_velocity")
    with solver(g, precision) as s:
        upload(s, g)
        s.advect_velocity(float(g["dt"]))
        for k in "uvw":
            out = s.download(k)
            ref, inp = g["out_" + k], g[k]
            scale = max(np.abs(inp).max(), 1.0)
            assert np.abs(out - ref).max() <= tol * scale, (k, np.abs(out - ref).max())
            # the fixed centre line and the faces outside the pipe keep their value
            keep = g["fixed_" + k] | (ref == inp)
            assert np.abs(out[keep] - inp[keep]).max() <= (0.0 if precision == fs.FS_PRECISION_FP64 else 1e-6)
        # the level set is not touched
        assert np.abs(s.download("phi") - g["phi"]).max() <= (0.0 if precision == fs.FS_PRECISION_FP64 else 1e-6)


def test_pipe_mode_refuses_the_operators_it_does_not_build():
    g = load("pipe_levelset")
    with solver(g) as s:
        upload(s, g)
        for call in (lambda: s.viscosity(1e-3),):
            with pytest.raises(fs.FsError) as e:
                call()
            assert e.value.status == fs.FS_NOT_SUPPORTED
        # the context stays usable
        s.advect_levelset(float(g["dt"]))
        assert np.isfinite(s.download("phi")).all()


def test_pipe_geometry_is_checked():
    g = load("pipe_levelset")
    n = tuple(int(x) for x in g["n"])
    # a pipe that reaches the box's ghost layers
    with pytest.raises(fs.FsError) as e:
        fs.Solver(n, 0.25, pipe=1, pipe_radius=2.45, grid_min=tuple(g["lo"]), grid_max=tuple(g["hi"]), pipe_R1=1.0,
                  pipe_V0=1.0, pipe_f=1.0, pipe_eta=1.1, pipe_oil_density=0.9, pipe_We=1.0)
    assert e.value.status == fs.FS_INVALID_ARG
    # grid_min/grid_max that do not give the grid's dx
    with pytest.raises(fs.FsError):
        fs.Solver(n, 0.2, pipe=1, pipe_radius=1.61, grid_min=tuple(g["lo"]), grid_max=tuple(g["hi"]), pipe_R1=1.0,
                  pipe_V0=1.0, pipe_f=1.0, pipe_eta=1.1, pipe_oil_density=0.9, pipe_We=1.0)


@pytest.mark.parametrize("precision", [fs.FS_PRECISION_FP64, fs.FS_PRECISION_FP32_REFINE])
def test_pipe_projection_matches_reference(precision):
    """EULERIAN_FLUID_SOLVER_3D::Projection of the pipe (fixture
    pipe_projection): Neumann cells outside the cylinder, the divergence of
    the pipe's velocity copies, the jump kappa/We, the deflated system solved
    to the reference's absolute r.z < tol^2, the pipe's velocity update with
    its fixed centre line and periodic rows.  FP64: the divergence to
    rounding, the PCG iterations within 2, pressure and velocities to 1e-9 of
    their scale; FP32 + refinement (the same system solved to the
    equivalent relative residual): pressure and velocities to 1e-5."""
    g = load("pipe_projection")
    fp64 = precision == fs.FS_PRECISION_FP64
    flags = fs.FS_FLAG_REINIT_TYPO | fs.FS_FLAG_FAITHFUL_PROJECTION | fs.FS_FLAG_CURVATURE_TYPO
    kw = dict(stop=fs.FS_STOP_ABSOLUTE, tolerance=float(g["tolerance"])) if fp64 else dict(tolerance=1e-9)
    with solver(g, precision, flags=flags, max_iteration=int(g["max_iteration"]), **kw) as s:
        upload(s, g)
        rep = s.project(float(g["dt"]))
        p = s.download("pressure")
        div = s.download("divergence")
        vel = {k: s.download(k) for k in "uvw"}
    fl = g["boundary"] <= 0
    assert fl.sum() == len(g["b_rows"])
    dscale = np.abs(g["div"]).max()
    assert np.abs(div - g["div"]).max() <= (1e-12 if fp64 else 1e-5) * dscale
    if fp64:
        assert abs(rep["iterations"] - int(g["iterations"])) <= 2
    pscale = np.abs(g["out_p"]).max()
    ptol = 1e-9 if fp64 else 1e-5
    assert np.abs(p[fl] - g["x_rows"]).max() <= ptol * pscale
    # the cells outside the pipe are no unknowns: their pressure stays 0
    assert np.abs(p[~fl]).max() == 0.0
    for k in "uvw":
        ref, inp = g["out_" + k], g[k]
        scale = max(np.abs(ref - inp).max(), 1.0)
        assert np.abs(vel[k] - ref).max() <= ptol * scale, (k, np.abs(vel[k] - ref).max())


def test_pipe_projection_matches_oracle_corrected_system():
    """The corrected pipe projection (the singular consistent system, no
    deflation) against the oracle's, FP64, solved to 1e-10 relative."""
    g = load("pipe_projection")
    grids = O.pipe_grids(tuple(int(x) for x in g["n"]), tuple(g["lo"]), tuple(g["hi"]))
    C = {k: float(g[k]) for k in ("a", "R1", "m", "eta", "K", "g", "f", "A", "V0", "J", "Re", "We")}
    fixed = (g["fixed_u"], g["fixed_v"], g["fixed_w"])
    u, v, w, p, info = O.pipe_projection(g["phi"], g["u"], g["v"], g["w"], grids, C, float(g["dt"]), 1e-12, 20000,
                                         float(g["water_density"]), float(g["oil_density"]), fixed=fixed,
                                         mode="corrected", criterion="rel")
    flags = fs.FS_FLAG_REINIT_TYPO | fs.FS_FLAG_CURVATURE_TYPO
    with solver(g, flags=flags, tolerance=1e-12, max_iteration=20000) as s:
        upload(s, g)
        s.project(float(g["dt"]))
        got = {k: s.download(k) for k in ("u", "v", "w", "pressure")}
    fl = info["fluid"]
    # the singular system's pressure is fixed up to a constant
    dp = (got["pressure"] - p)[fl]
    assert np.abs(dp - dp.mean()).max() <= 1e-8 * np.abs(p[fl]).max()
    for k, ref in zip("uvw", (u, v, w)):
        assert np.abs(got[k] - ref).max() <= 1e-8 * max(np.abs(ref - g[k]).max(), 1.0), k


@pytest.mark.parametrize("precision,tol", [(fs.FS_PRECISION_FP64, 1e-14), (fs.FS_PRECISION_FP32_REFINE, 1e-6)])
def test_pipe_cfl_matches_reference(precision, tol):
    """CFLOneTimeStep of the pipe on the projected velocities of fixture
    pipe_projection, with the curvature maximum of its level set (the
    reference's comes from the projection just run on the same level set)."""
    g = load("pipe_projection")
    with solver(g, precision, flags=fs.FS_FLAG_REINIT_TYPO | fs.FS_FLAG_CURVATURE_TYPO, cfl=1.0) as s:
        s.upload("phi", g["phi"])
        for k in "uvw":
            s.upload(k, g["out_" + k])
        dt = s.cfl_dt()
    assert abs(dt - float(g["cfl"])) <= tol * float(g["cfl"])


@pytest.mark.parametrize("precision,tol", [(fs.FS_PRECISION_FP64, 1e-9), (fs.FS_PRECISION_FP32_REFINE, 5e-4)])
def test_pipe_frame_matches_reference(precision, tol):
    """One whole SIMULATION_WORLD::AdvanceOneFrame of the pipe with the
    sourcing step off (fixture pipe_frame): fs_cfl_dt times the script's CFL
    gives the reference's dt, then fs_step (order 2: level-set Heun, velocity
    Heun over ENO3 advection + body force + projection, reinitialisation
    Heun).  Fields to `tol` of their maximum: 1e-9 in FP64 (the PCG stops at
    the reference's absolute r.z < tol^2 within an iteration or two of it),
    5e-4 with FP32 storage; the pressure on the unknowns likewise."""
    g = load("pipe_frame")
    fp64 = precision == fs.FS_PRECISION_FP64
    flags = fs.FS_FLAG_REINIT_TYPO | fs.FS_FLAG_FAITHFUL_PROJECTION | fs.FS_FLAG_CURVATURE_TYPO
    kw = dict(stop=fs.FS_STOP_ABSOLUTE, tolerance=float(g["tolerance"])) if fp64 else dict(tolerance=1e-9)
    with solver(g, precision, flags=flags, order=2, cfl=float(g["cfl_number"]),
                max_iteration=int(g["max_iteration"]), **kw) as s:
        upload(s, g)
        dt = s.cfl_dt()
        assert abs(dt - float(g["dt"])) <= (1e-14 if fp64 else 1e-6) * float(g["dt"])
        s.step(float(g["dt"]))
        got = {k: s.download(k) for k in ("phi", "u", "v", "w", "pressure")}
    for k in ("phi", "u", "v", "w"):
        ref = g["out_" + k]
        assert np.abs(got[k] - ref).max() <= tol * np.abs(ref).max(), (k, np.abs(got[k] - ref).max())
    fl = g["boundary"] <= 0
    ref = g["out_p"]
    assert np.abs(got["pressure"][fl] - ref[fl]).max() <= tol * np.abs(ref).max()


def test_pipe_step_refuses_viscosity():
    g = load("pipe_frame")
    with solver(g, viscosity=1) as s:
        upload(s, g)
        with pytest.raises(fs.FsError) as e:
            s.step(1e-3)
        assert e.value.status == fs.FS_NOT_SUPPORTED


def test_pipe_script_frame_matches_reference(tmp_path):
    """The drop-in path: the reference's pipe script (sourcing off) read by
    EULERIAN_FLUID_SOLVER_3D.FromScript, the fixture's fields set, the CFL dt
    and one AdvanceOneTimeStepThread against the reference's frame."""
    from fluid_simulator_backup_b200 import reference_api as R
    from oracle import refsim
    g = load("pipe_frame")
    n = tuple(int(x) for x in g["n"])
    path = refsim.write_pipe_sim(str(tmp_path / "pipe.sim"), n, tuple(g["lo"]), tuple(g["hi"]), sourcing=False)
    s = R.EULERIAN_FLUID_SOLVER_3D.FromScript(path)
    try:
        s.water_levelset = g["phi"]
        s.set_velocity(g["u"], g["v"], g["w"])
        dt = s.CFLOneTimeStep() * s.solver.params.cfl
        assert abs(dt - float(g["dt"])) <= 1e-14 * float(g["dt"])
        s.AdvanceOneTimeStepThread(0, float(g["dt"]))
        assert np.abs(s.water_levelset - g["out_phi"]).max() <= 1e-9 * np.abs(g["out_phi"]).max()
        for k, a in zip("uvw", s.velocity()):
            assert np.abs(a - g["out_" + k]).max() <= 1e-9 * np.abs(g["out_" + k]).max(), k
    finally:
        s.solver.close()
