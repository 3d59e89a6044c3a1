"""The C++ host mirror (include/fluid_b200_solver.hpp), built with g++ and
driven by tests/cpp/mirror_main.cpp.

- on CPU: the header compiles, and the C++ .sim reader maps a script to the
  same fs_params as the Python mirror;
- on the GPU: CUDA_PCG_METHOD (through the LINEAR_SOLVER base, worker
  threads returning at once) reproduces the reference's own PCG solution of a
  projection system, and EULERIAN_FLUID_SOLVER_3D built from a script steps
  bit-identically to the Python mirror on the same library.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import fluid_simulator_backup_b200 as fs
from fluid_simulator_backup_b200.reference_api import GRID_STRUCTURE_3D, EULERIAN_FLUID_SOLVER_3D, params_from_block
from fluid_simulator_backup_b200.script import SCRIPT_READER

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "fluid_simulator_backup_b200")


@pytest.fixture(scope="module")
def mirror(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    fs.lib()  # the library must exist before linking against it
    out = str(tmp_path_factory.mktemp("cpp") / "mirror")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "mirror_main.cpp"), "-o", out, "-L", PKG, "-lfluidb200",
           "-Wl,-rpath," + PKG]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


def write_script(path, n, **kw):
    from oracle.refsim import write_sim
    return write_sim(path, n, water_drop=False, **kw)


def test_cpp_script_reader_matches_python(mirror, tmp_path):
    path = write_script(str(tmp_path / "box.sim"), 24, tolerance=1e-9, max_iteration=777, reinit_iterations=7,
                        cfl=0.6, order=2)
    out = subprocess.run([mirror, "script", path], check=True, capture_output=True, text=True).stdout.split()

    def after(key, k=1):
        return out[out.index(key) + k]
    vals = {key: after(key) for key in ("dx", "tol", "maxit", "stop", "order", "cfl")}
    r = SCRIPT_READER(path)
    g = GRID_STRUCTURE_3D().InitializeFromBlock(
        r.FindBlock("SIMULATION_WORLD").FindBlock("WORLD_DISCRETIZATION_AIR_WATER").FindBlock("GRID_STRUCTURE_3D_LARGE"))
    p = params_from_block(r.FindBlock("FLUID_SOLVER_UNIFORM_AIR_WATER"), g)
    assert out[0] == "res" and out[1:4] == ["24", "24", "24"]
    assert float(vals["dx"]) == g.dx
    i = out.index("rho")
    assert (float(out[i + 1]), float(out[i + 2])) == (p.rho_neg, p.rho_pos)
    assert (float(out[i + 4]), float(out[i + 5])) == (p.mu_neg, p.mu_pos)
    assert float(vals["tol"]) == p.tolerance and int(vals["maxit"]) == p.max_iteration == 777
    assert int(vals["stop"]) == p.stop and int(vals["order"]) == p.order == 2
    i = out.index("reinit")
    assert (int(out[i + 1]), int(out[i + 2])) == (p.reinit_iterations, p.reinit_scaling) == (7, 5)
    assert float(vals["cfl"]) == 0.6


@pytest.mark.gpu
def test_cpp_linear_solver_plugin_reproduces_reference_pcg(mirror, tmp_path):
    g = np.load(os.path.join(ROOT, "tests", "golden", "projection_bubble.npz"))
    vals, cols, rp, b = g["csr_vals"], g["csr_cols"].astype(np.int32), g["csr_rowptr"].astype(np.int32), g["b"]
    prob = tmp_path / "prob.bin"
    with open(prob, "wb") as f:
        np.array([len(b), len(vals)], np.int32).tofile(f)
        np.array([float(g["tol"])], np.float64).tofile(f)
        np.array([100000], np.int32).tofile(f)
        vals.astype(np.float64).tofile(f)
        cols.tofile(f)
        rp.tofile(f)
        b.astype(np.float64).tofile(f)
    out = tmp_path / "x.bin"
    res = subprocess.run([mirror, "csr", str(prob), str(out)], check=True, capture_output=True, text=True).stdout.split()
    x = np.fromfile(out, np.float64)
    assert abs(int(res[1]) - int(g["iterations"])) <= 2
    assert np.linalg.norm(x - g["x"]) / np.linalg.norm(g["x"]) < 1e-7


@pytest.mark.gpu
def test_cpp_solver_steps_like_the_python_mirror(mirror, tmp_path):
    n = 16
    path = write_script(str(tmp_path / "bubble.sim"), n, tolerance=1e-10, order=3)
    x = (np.arange(n) + 0.5) / n
    phi = np.sqrt((x[None, None, :] - 0.5) ** 2 + (x[None, :, None] - 0.35) ** 2 + (x[:, None, None] - 0.5) ** 2) - 0.2
    phi_in = tmp_path / "phi.bin"
    phi.astype(np.float64).tofile(phi_in)
    phi_out = tmp_path / "phi_out.bin"
    res = subprocess.run([mirror, "step", path, str(phi_in), str(phi_out)], check=True, capture_output=True,
                         text=True).stdout.split()
    got = np.fromfile(phi_out, np.float64).reshape(n, n, n)
    s = EULERIAN_FLUID_SOLVER_3D.FromScript(path)
    s.water_levelset = phi
    s.set_velocity(np.zeros((n, n, n + 1)), np.zeros((n, n + 1, n)), np.zeros((n + 1, n, n)))
    dt = s.solver.params.cfl * s.CFLOneTimeStep()
    assert float(res[1]) == dt
    s.AdvanceOneTimeStepThread(0, dt)
    want = s.water_levelset
    s.solver.close()
    assert int(res[5]) in (fs.FS_OK, fs.FS_NOT_CONVERGED)
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_cpp_levelset_mirror_sweeps_and_writes_obj_like_python(mirror, tmp_path):
    """FullFastSweepingMethodThreaded and WRITE_LEVELSET::WriteOBJ through the
    C++ mirror give the Python mirror's level set and the same OBJ bytes."""
    from fluid_simulator_backup_b200.reference_api import WRITE_LEVELSET
    n = 16
    path = write_script(str(tmp_path / "ls.sim"), n)
    x = (np.arange(n) + 0.5) / n
    phi = 1.4 * (np.sqrt((x[None, None, :] - 0.5) ** 2 + (x[None, :, None] - 0.4) ** 2
                         + (x[:, None, None] - 0.5) ** 2) - 0.25)
    phi_in = tmp_path / "phi.bin"
    phi.astype(np.float64).tofile(phi_in)
    out_phi, out_obj = tmp_path / "phi_out.bin", tmp_path / "cpp.obj"
    subprocess.run([mirror, "levelset", path, str(phi_in), str(out_phi), str(out_obj)], check=True,
                   capture_output=True, text=True)
    s = EULERIAN_FLUID_SOLVER_3D.FromScript(path)
    s.water_levelset = phi
    s.FullFastSweepingMethodThreaded()
    py_obj = tmp_path / "py.obj"
    WRITE_LEVELSET(s).WriteOBJ(str(py_obj))
    want = s.water_levelset
    s.solver.close()
    assert np.array_equal(np.fromfile(out_phi, np.float64).reshape(n, n, n), want)
    assert open(out_obj).read() == open(py_obj).read()
    from oracle import fs_oracle as O
    assert np.array_equal(want, O.fast_sweeping(phi, s.base_grid.dx, 3))  # each call starts from its own set-up


def test_pipe_mode_scripts_are_refused(mirror, tmp_path):
    """A box script switched to the reference's oil/water pipe mode (no pipe
    blocks, so no vertical pipe) is refused by both script readers instead of
    being run as a box."""
    path = write_script(str(tmp_path / "pipe.sim"), 16)
    text = open(path).read()
    assert "oil_water_simulation = false" in text
    with open(path, "w") as f:
        f.write(text.replace("air_water_simulation = true", "air_water_simulation = false")
                .replace("oil_water_simulation = false", "oil_water_simulation = true"))
    with pytest.raises(ValueError):
        EULERIAN_FLUID_SOLVER_3D.FromScript(path)
    res = subprocess.run([mirror, "step", path, "/dev/null", str(tmp_path / "out.bin")], capture_output=True,
                         text=True)
    assert res.returncode != 0 and "pipe mode" in res.stderr


def test_cpp_pipe_reader_gives_the_reference_constants(mirror, tmp_path):
    """The C++ mirror's pipe reader (pipe_params_from_script) derives the
    reference's dimensionless constants bit for bit (fixture pipe_frame, made
    by the reference) and refuses a script with the sourcing step on."""
    from oracle.refsim import write_pipe_sim
    g = dict(np.load(os.path.join(ROOT, "tests", "golden", "pipe_frame.npz")))
    n = tuple(int(x) for x in g["n"])
    path = write_pipe_sim(str(tmp_path / "pipe.sim"), n, tuple(g["lo"]), tuple(g["hi"]), sourcing=False)
    out = subprocess.run([mirror, "pipe_script", path], check=True, capture_output=True, text=True).stdout.split()
    val = {out[q]: out[q + 1] for q in range(0, len(out), 2)}
    assert int(val["pipe"]) == 1 and int(val["viscosity"]) == 0 and int(val["order"]) == 2
    for key, ref in (("radius", "a"), ("R1", "R1"), ("V0", "V0"), ("f", "f"), ("eta", "eta"), ("We", "We"),
                     ("oil", "oil_density")):
        assert float(val[key]) == float(g[ref]), key
    assert float(val["rho_pos"]) == float(g["water_density"]) / float(g["oil_density"])
    path = write_pipe_sim(str(tmp_path / "pipe_on.sim"), n, tuple(g["lo"]), tuple(g["hi"]), sourcing=True)
    res = subprocess.run([mirror, "pipe_script", path], capture_output=True, text=True)
    assert res.returncode != 0 and "is_sourcing_active" in res.stderr
