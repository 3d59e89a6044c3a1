"""Fast sweeping reinitialisation (LEVELSET_3D::ReinitializeByFastSweeping,
LEVELSET_3D.h:601-610, 734-918) through the C ABI.

- on CPU: fastsweeping_reinitialization / sussmanstyle_reinitialization map
  to fs_params in the Python and C++ script readers;
- on the GPU: the hyperplane sweeps against the oracle's sequential
  Gauss-Seidel sweeps bit for bit in FP64 (every sweep direction, the
  reference's single call and the corrected full method, a box that is not a
  cube), FP32 to its rounding, the reference's own output (golden, with its
  sort defect and the NaNs it writes) through FS_FLAG_SORT_TYPO, the sweep
  counter, and a whole step with fast sweeping against the oracle step.
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


def noisy_sphere(n, seed, scale=1.5, noise=0.01):
    nx, ny, nz = n
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / nx
    z = (np.arange(nz) + 0.5) / nx
    sd = np.sqrt((x[None, None, :] - 0.5) ** 2 + (y[None, :, None] - 0.45) ** 2 + (z[:, None, None] - 0.4) ** 2) - 0.3
    return sd * scale + np.random.default_rng(seed).normal(size=sd.shape) * noise


def script_params(path):
    r = SCRIPT_READER(path)
    g = GRID_STRUCTURE_3D().InitializeFromBlock(
        r.FindBlock("SIMULATION_WORLD").FindBlock("WORLD_DISCRETIZATION_AIR_WATER").FindBlock("GRID_STRUCTURE_3D_LARGE"))
    return params_from_block(r.FindBlock("FLUID_SOLVER_UNIFORM_AIR_WATER"), g)


@pytest.mark.parametrize("fast,sussman", [(False, True), (True, True), (True, False), (False, False)])
def test_script_selects_the_reinitialisation(tmp_path, fast, sussman):
    path = write_sim(str(tmp_path / "box.sim"), 16, water_drop=False, fast_sweeping=fast, sussman=sussman,
                     reinit_iterations=7)
    p = script_params(path)
    assert p.fast_sweeping == int(fast)
    assert p.reinit_iterations == (7 if sussman else 0)
    if shutil.which("g++") is None:
        return
    fs.lib()
    exe = str(tmp_path / "mirror")
    pkg = os.path.join(ROOT, "fluid_simulator_backup_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "mirror_main.cpp"), "-o", exe, "-L", pkg, "-lfluidb200",
                    "-Wl,-rpath," + pkg], check=True, capture_output=True, text=True)
    out = subprocess.run([exe, "script", path], check=True, capture_output=True, text=True).stdout.split()
    assert int(out[out.index("fast_sweeping") + 1]) == int(fast)
    assert int(out[out.index("reinit_iterations") + 1]) == p.reinit_iterations


def run_gpu(phi, dx, direction, pairs=1, precision=fs.FS_PRECISION_FP64, flags=0):
    nz, ny, nx = phi.shape
    with fs.Solver((nx, ny, nz), dx, precision=precision, flags=flags) as s:
        s.upload("phi", phi)
        s.fast_sweeping(direction, pairs)
        return s.download("phi")


@pytest.mark.gpu
@pytest.mark.parametrize("direction", [0, 1, 2, 3])
def test_hyperplane_sweeps_match_the_sequential_sweeps(direction):
    """The parallel hyperplane order reads what the sequential sweep reads:
    FP64 results are identical bit for bit."""
    n = (18, 22, 16)
    phi = noisy_sphere(n, direction)
    dx = 1.0 / n[0]
    np.testing.assert_array_equal(run_gpu(phi, dx, direction), O.fast_sweeping(phi, dx, direction))


@pytest.mark.gpu
def test_full_method_matches_the_oracle_and_the_distance():
    n = (24, 24, 24)
    phi = noisy_sphere(n, 7, scale=1.7, noise=0.0)
    dx = 1.0 / 24
    got = run_gpu(phi, dx, 2, pairs=4)
    np.testing.assert_array_equal(got, O.fast_sweeping(phi, dx, 2, pairs=4))
    sd = noisy_sphere(n, 7, scale=1.0, noise=0.0)
    band = np.abs(sd) < 0.3
    assert np.abs(got - sd)[band].max() < dx


@pytest.mark.gpu
def test_fp32_fast_sweeping_matches_the_oracle():
    n = (20, 20, 20)
    phi = noisy_sphere(n, 11)
    dx = 1.0 / 20
    got = run_gpu(phi, dx, 1, precision=fs.FS_PRECISION_FP32_REFINE)
    ref = O.fast_sweeping(phi, dx, 1)
    assert np.abs(got - ref).max() < 1e-5 * np.abs(ref).max()


@pytest.mark.gpu
def test_golden_fast_sweeping_through_cuda():
    """The reference's own output, NaNs included, with its sort as written."""
    g = dict(np.load(os.path.join(GOLD, "fast_sweeping.npz")))
    for direction in (0, 3):
        got = run_gpu(g["phi"], float(g["dx"]), direction, flags=fs.FS_FLAG_SORT_TYPO)
        np.testing.assert_array_equal(got, g[f"out_{direction}"])


@pytest.mark.gpu
def test_sort_typo_reports_the_uninitialised_read():
    """An input on which the reference's sort reads a2 before the sweep ever
    wrote it (the oracle says which) is refused instead of inventing a value."""
    n = (20, 20, 20)
    for seed in range(4, 40):
        phi = noisy_sphere(n, seed)
        try:
            O.fast_sweeping(phi, 1.0 / 20, 1, typo=True)
        except ValueError:
            break
    else:
        pytest.skip("no input found that reads the uninitialised value")
    with pytest.raises(fs.FsError) as e:
        run_gpu(phi, 1.0 / 20, 1, flags=fs.FS_FLAG_SORT_TYPO)
    assert e.value.status == fs.FS_NONFINITE


@pytest.mark.gpu
def test_sweep_counter_advances_like_the_reference():
    n = (16, 16, 16)
    phi = noisy_sphere(n, 13)
    dx = 1.0 / 16
    with fs.Solver(n, dx) as s:
        s.upload("phi", phi)
        for _ in range(3):
            s.fast_sweeping()
        got = s.download("phi")
    ref = phi
    for d in range(3):
        ref = O.fast_sweeping(ref, dx, d)
    np.testing.assert_array_equal(got, ref)


@pytest.mark.gpu
def test_whole_step_with_fast_sweeping_matches_oracle():
    n = 16
    dx = 1.0 / n
    x = (np.arange(n) + 0.5) / n
    phi = np.sqrt((x[None, None, :] - 0.5) ** 2 + (x[None, :, None] - 0.35) ** 2 + (x[:, None, None] - 0.5) ** 2) - 0.2
    u = np.zeros((n, n, n + 1)); v = np.zeros((n, n + 1, n)); w = np.zeros((n + 1, n, n))
    P = dict(rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, gravity=(0.0, -9.8, 0.0), eps=1e-6,
             reinit_iterations=4, reinit_scaling=5, tol=1e-12, max_iter=20000, viscosity=True, visc_tol=1e-12,
             fast_sweeping=True)
    with fs.Solver(n, dx, rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, tolerance=1e-12,
                   stop=fs.FS_STOP_RELATIVE, viscosity_tolerance=1e-12, reinit_iterations=4, fast_sweeping=1) as s:
        for k, a in zip(("phi", "u", "v", "w"), (phi, u, v, w)):
            s.upload(k, a)
        dt = s.cfl_dt()
        s.step(dt)
        got = [s.download(k) for k in ("phi", "u", "v", "w")]
    ref = O.step(phi, u, v, w, dx, dt, P)
    for a, b in zip(got, ref[:4]):
        assert np.abs(a - b).max() < 1e-8 * max(np.abs(b).max(), 1e-3)
    assert ref[5]["sweep_direction"] == 3
