"""ENO3 velocity self-advection (the reference's VELOCITY_ADVECTION
use_3rd_eno_v, ADVECTION_3D.h:323-325, ADVECTION_METHOD_3D.h:1639-1934).

- on CPU: a script that selects ENO3 maps to FS_VELOCITY_ENO3 in the Python
  and C++ mirrors of the .sim reader;
- on the GPU: the kernel against the oracle (FP64 to 1e-10, FP32 storage to
  2e-5), against the reference's own ENO3 output (golden), a whole step with
  ENO3 against the oracle step, and the adjoint entry refusing ENO3.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import fluid_simulator_backup_b200 as fs
from fluid_simulator_backup_b200.reference_api import GRID_STRUCTURE_3D, params_from_block
from fluid_simulator_backup_b200.script import SCRIPT_READER
from oracle import fs_oracle as O
from oracle.refsim import write_sim

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def random_velocity(n, seed, scale=0.3):
    rng = np.random.default_rng(seed)
    nx, ny, nz = n
    return (rng.normal(size=(nz, ny, nx + 1)) * scale, rng.normal(size=(nz, ny + 1, nx)) * scale,
            rng.normal(size=(nz + 1, ny, nx)) * scale)


def eno3_solver(n, precision=fs.FS_PRECISION_FP64, **kw):
    if isinstance(n, int):
        n = (n, n, n)
    return fs.Solver(n, 1.0 / n[0], precision=precision, velocity_scheme=fs.FS_VELOCITY_ENO3, **kw)


def script_params(path):
    r = SCRIPT_READER(path)
    g = GRID_STRUCTURE_3D().InitializeFromBlock(
        r.FindBlock("SIMULATION_WORLD").FindBlock("WORLD_DISCRETIZATION_AIR_WATER").FindBlock("GRID_STRUCTURE_3D_LARGE"))
    return params_from_block(r.FindBlock("FLUID_SOLVER_UNIFORM_AIR_WATER"), g)


def test_script_selects_eno3(tmp_path):
    for weno, want in ((True, fs.FS_VELOCITY_WENO5), (False, fs.FS_VELOCITY_ENO3)):
        path = write_sim(str(tmp_path / "box.sim"), 16, water_drop=False, velocity_weno=weno, epsilon=2e-6)
        p = script_params(path)
        assert p.velocity_scheme == want
        assert p.velocity_epsilon == 2e-6
    # both schemes selected: the reference would advect twice in one stage
    text = open(path).read().replace("use_5th_weno_v = false", "use_5th_weno_v = true")
    with open(path, "w") as f:
        f.write(text)
    with pytest.raises(ValueError):
        script_params(path)


def test_cpp_script_reader_selects_eno3(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    fs.lib()
    exe = str(tmp_path / "mirror")
    pkg = os.path.join(ROOT, "fluid_simulator_backup_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "mirror_main.cpp"), "-o", exe, "-L", pkg, "-lfluidb200",
                    "-Wl,-rpath," + pkg], check=True, capture_output=True, text=True)
    for weno, want in ((True, fs.FS_VELOCITY_WENO5), (False, fs.FS_VELOCITY_ENO3)):
        path = write_sim(str(tmp_path / "box.sim"), 16, water_drop=False, velocity_weno=weno, epsilon=2e-6)
        out = subprocess.run([exe, "script", path], check=True, capture_output=True, text=True).stdout.split()
        assert int(out[out.index("velocity_scheme") + 1]) == want
        assert float(out[out.index("velocity_epsilon") + 1]) == 2e-6
    text = open(path).read().replace("use_5th_weno_v = false", "use_5th_weno_v = true")
    with open(path, "w") as f:
        f.write(text)
    assert subprocess.run([exe, "script", path], capture_output=True, text=True).returncode != 0


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(fs.FS_PRECISION_FP64, 1e-10), (fs.FS_PRECISION_FP32_REFINE, 2e-5)])
def test_eno3_velocity_matches_oracle(precision, tol):
    n = (16, 18, 14)
    u, v, w = random_velocity(n, 7)
    with eno3_solver(n, precision) as s:
        for k, a in zip("uvw", (u, v, w)):
            s.upload(k, a)
        s.advect_velocity(2e-3)
        got = [s.download(k) for k in "uvw"]
    ref = O.eno3_velocity(u, v, w, 1.0 / n[0], 2e-3)
    for g, r in zip(got, ref):
        assert rel_err(g, r) < tol


@pytest.mark.gpu
def test_golden_eno3_through_cuda():
    g = dict(np.load(os.path.join(GOLD, "eno3_velocity.npz")))
    n = int(g["n"])
    with fs.Solver((n, n, n), float(g["dx"]), velocity_scheme=fs.FS_VELOCITY_ENO3) as s:
        for k in "uvw":
            s.upload(k, g[k])
        s.advect_velocity(float(g["dt"]))
        for k in "uvw":
            assert rel_err(s.download(k), g["out_" + k]) < 1e-10


@pytest.mark.gpu
def test_whole_step_with_eno3_matches_oracle():
    n = 16
    dx = 1.0 / n
    x = (np.arange(n) + 0.5) / n
    phi = np.sqrt((x[None, None, :] - 0.5) ** 2 + (x[None, :, None] - 0.35) ** 2 + (x[:, None, None] - 0.5) ** 2) - 0.2
    u, v, w = random_velocity((n, n, n), 8, scale=0.05)
    u[:, :, 0] = u[:, :, -1] = 0; v[:, 0, :] = v[:, -1, :] = 0; w[0] = w[-1] = 0
    P = dict(rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, gravity=(0.0, -9.8, 0.0), eps=1e-6,
             reinit_iterations=10, reinit_scaling=5, tol=1e-12, max_iter=20000, viscosity=True, visc_tol=1e-12,
             velocity_eno3=True)
    with eno3_solver(n, rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, tolerance=1e-12,
                     stop=fs.FS_STOP_RELATIVE, viscosity_tolerance=1e-12) as s:
        for k, a in zip(("phi", "u", "v", "w"), (phi, u, v, w)):
            s.upload(k, a)
        dt = s.cfl_dt()
        s.step(dt)
        got = [s.download(k) for k in ("phi", "u", "v", "w")]
    ref = O.step(phi, u, v, w, dx, dt, P)
    for a, b in zip(got, ref[:4]):
        assert rel_err(a, b) < 1e-8
    # and it is not the WENO5 step
    ref5 = O.step(phi, u, v, w, dx, dt, dict(P, velocity_eno3=False))
    assert rel_err(got[1], ref5[1]) > 1e-6


@pytest.mark.gpu
def test_adjoint_refuses_eno3():
    n = 12
    with eno3_solver(n) as s:
        with pytest.raises(fs.FsError) as e:
            s.adjoint_reset()
            s.step_adjoint(1e-3)
        assert e.value.status == fs.FS_NOT_SUPPORTED
