"""Oil/water vertical pipe mode through the CUDA path against the reference's
own outputs (fixtures pipe_*, made by tests/golden/make_golden.py from the
headless reference build) and against the oracle.

The pipe mode's level-set advection, reinitialisation, ENO3 velocity
advection and dimensionless body force run on the GPU; its viscosity and
projection are not built, and those entry points (and fs_step) return
FS_NOT_SUPPORTED in this mode."""
import os

import numpy as np
import pytest

import fluid_simulator_backup_b200 as fs
from oracle import fs_oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def solver(g, precision=fs.FS_PRECISION_FP64, flags=fs.FS_FLAG_REINIT_TYPO):
    n = tuple(int(x) for x in g["n"])
    dx = (float(g["hi"][0]) - float(g["lo"][0])) / (n[0] - 1)
    return fs.Solver(n, dx, precision=precision, pipe=1, pipe_radius=float(g["a"]), grid_min=tuple(g["lo"]),
                     grid_max=tuple(g["hi"]), pipe_R1=float(g["R1"]), pipe_V0=float(g["V0"]), pipe_f=float(g["f"]),
                     pipe_eta=float(g["eta"]), pipe_oil_density=float(g["oil_density"]),
                     gravity=(0.0, float(g["gravity_y"]), 0.0), weno_epsilon=float(g["epsilon"]),
                     reinit_iterations=int(g["reinit_iterations"]), reinit_scaling=int(g["reinit_scaling"]),
                     flags=flags, viscosity=0, velocity_scheme=fs.FS_VELOCITY_ENO3)


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
        for call in (lambda: s.step(1e-3), lambda: s.project(1e-3), lambda: s.viscosity(1e-3),
                     lambda: s.cfl_dt()):
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
                  pipe_V0=1.0, pipe_f=1.0, pipe_eta=1.1, pipe_oil_density=0.9)
    assert e.value.status == fs.FS_INVALID_ARG
    # grid_min/grid_max that do not give the grid's dx
    with pytest.raises(fs.FsError):
        fs.Solver(n, 0.2, pipe=1, pipe_radius=1.61, grid_min=tuple(g["lo"]), grid_max=tuple(g["hi"]), pipe_R1=1.0,
                  pipe_V0=1.0, pipe_f=1.0, pipe_eta=1.1, pipe_oil_density=0.9)
