"""CPU checks of the drop-in boundary: the C-ABI library is built, loads and
exports every entry point include/fluid_b200.h declares; host-side logic
(script reader, parameter mapping, argument validation) works without a GPU.
No compute call is made here."""
import ctypes
import os
import re

import numpy as np
import pytest

import fluid_simulator_backup_b200 as fs
from fluid_simulator_backup_b200 import reference_api as ra
from fluid_simulator_backup_b200.script import SCRIPT_READER, ScriptError

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "fluid_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fs_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = fs.lib()
    names = declared_symbols()
    assert len(names) >= 19
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(fs.EXPORTED)


def test_params_default_and_status_strings():
    p = fs.default_params()
    assert p.order == 3 and p.reinit_iterations == 10 and p.reinit_scaling == 5
    assert p.gravity[1] == -9.8 and p.precision == fs.FS_PRECISION_FP64
    assert fs.status_str(fs.FS_NOT_CONVERGED) == "iterative solve not converged"
    assert fs.status_str(99) == "unknown status"


def test_create_rejects_bad_arguments_before_touching_the_device():
    L = fs.lib()
    h = ctypes.c_void_p()
    g = fs.GridDesc(2, 8, 8, 0.1)  # too small
    assert L.fs_create(ctypes.byref(g), None, ctypes.byref(h)) == fs.FS_INVALID_ARG
    g = fs.GridDesc(8, 8, 8, -1.0)
    assert L.fs_create(ctypes.byref(g), None, ctypes.byref(h)) == fs.FS_INVALID_ARG
    g = fs.GridDesc(8, 8, 8, 0.125)
    p = fs.default_params(order=5)
    assert L.fs_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)) == fs.FS_INVALID_ARG
    p = fs.default_params(rho_neg=-1.0)
    assert L.fs_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)) == fs.FS_INVALID_ARG
    assert "densities" in fs.last_error()
    assert L.fs_step(None, ctypes.c_double(0.1), None) == fs.FS_INVALID_ARG
    assert L.fs_destroy(None) == fs.FS_OK
    p = fs.default_params(velocity_scheme=7)
    assert L.fs_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)) == fs.FS_INVALID_ARG
    assert "velocity scheme" in fs.last_error()
    p = fs.default_params(velocity_epsilon=-1.0)
    assert L.fs_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)) == fs.FS_INVALID_ARG
    # the reinitialisation and surface entry points refuse a missing context
    assert L.fs_fast_sweeping(None, 0, 1) == fs.FS_INVALID_ARG
    n64 = ctypes.c_int64()
    assert L.fs_surface(None, ctypes.byref(n64), ctypes.byref(n64)) == fs.FS_INVALID_ARG
    assert L.fs_surface_download(None, None, None, None) == fs.FS_INVALID_ARG
    assert L.fs_write_obj(None, b"x.obj") == fs.FS_INVALID_ARG


def test_pcg_csr_validates_the_matrix_on_the_host():
    # a row without a diagonal entry is rejected before any device work
    vals = np.array([1.0, 2.0]); cols = np.array([1, 0], dtype=np.int32); rp = np.array([0, 1, 2], dtype=np.int32)
    L = fs.lib()
    b = np.ones(2); x = np.zeros(2); it = ctypes.c_int(); res = ctypes.c_double()
    s = L.fs_pcg_csr(None, 2, 2, vals.ctypes.data, cols.ctypes.data, rp.ctypes.data, b.ctypes.data, x.ctypes.data,
                     1e-8, 10, 0, ctypes.byref(it), ctypes.byref(res))
    assert s == fs.FS_INVALID_ARG


def test_pcg_csr_noalloc_rejects_bad_arguments_on_the_host():
    # argument checks and the fixed-scratch row limit come before any device
    # work, so they answer without a GPU (the pointers are never dereferenced)
    L = fs.lib()
    fake = 256
    args = (fake, fake, fake, fake, fake, 1e-8, 10, fs.FS_STOP_RELATIVE, None, None, None)
    assert L.fs_pcg_csr_noalloc((1 << 18) + 1, 7, *args) == fs.FS_INVALID_ARG
    assert L.fs_pcg_csr_noalloc(0, 7, *args) == fs.FS_INVALID_ARG
    assert L.fs_pcg_csr_noalloc(8, 7, None, *args[1:]) == fs.FS_INVALID_ARG
    assert L.fs_pcg_csr_noalloc(8, 7, *args[:7], 5, None, None, None) == fs.FS_INVALID_ARG


@pytest.mark.parametrize("name", ["3D_script.sim", "3D_script_1.sim"])
def test_script_reader_reads_reference_scripts(name):
    ref = os.environ.get("FS_REFERENCE_DIR")
    if not ref or not os.path.exists(os.path.join(ref, name)):
        pytest.skip("FS_REFERENCE_DIR does not point at the reference's scripts")
    path = os.path.join(ref, name)
    r = SCRIPT_READER(path)
    b = r.FindBlock("FLUID_SOLVER_UNIFORM_AIR_WATER")
    assert b.GetFloat("water_density") == 1000.0
    assert b.GetVector3("gravity") == (0.0, -9.8, 0.0)
    assert b.FindBlock("PROJECTION_WATER").GetString("poisson_solver_type") == "PCG"
    assert b.GetFloat("missing_key", 7.0) == 7.0


def test_script_reader_syntax():
    text = """A { x = 0.5 flag = true v = (1, -2, 3.5) s = "PCG"
      // SKIPPED { y = 1 }
      B { n = 12 } /* c */ }"""
    r = SCRIPT_READER(text=text)
    a = r.FindBlock("A")
    assert a.GetFloat("x") == 0.5 and a.GetBoolean("flag") and a.GetVector3("v") == (1.0, -2.0, 3.5)
    assert a.GetString("s") == "PCG" and a.FindBlock("B").GetInteger("n") == 12
    assert a.FindBlock("SKIPPED").GetInteger("y", -1) == -1
    with pytest.raises(ScriptError):
        SCRIPT_READER(text="A { x = 1e-6 }").FindBlock("A").GetFloat("x")


def test_params_from_block_maps_reference_keys():
    text = """F { water_density = 1000 air_density = 1 water_viscosity = 0.001 air_viscosity = 0.000018
       order_for_time_advancing = 3 iteration_number_for_reinitialization = 10
       LEVELSET_ADVECTION { epsilon = 0.000001 }
       PROJECTION_WATER { tolerance = 0.00001 max_iteration = 500 air_bubble_rising = true water_drop = false
                          relative_tolerance = true } precision = "fp32_refine" }"""
    b = SCRIPT_READER(text=text).FindBlock("F")
    g = ra.GRID_STRUCTURE_3D((16, 16, 16), (0, 0, 0), (0, 0, 0), (15 / 16, 15 / 16, 15 / 16))
    p = ra.params_from_block(b, g)
    assert p.rho_neg == 1.0 and p.rho_pos == 1000.0  # bubble: air at phi <= 0
    assert p.order == 3 and p.max_iteration == 500 and abs(p.tolerance - 1e-5) < 1e-20
    assert p.precision == fs.FS_PRECISION_FP32_REFINE and p.stop == fs.FS_STOP_RELATIVE
    assert abs(g.dx - 1 / 16) < 1e-15


def test_solver_settings_are_checked_on_the_host():
    """The pressure preconditioner, reliable-update factor and flux
    arithmetic are fs_params fields, checked by fs_create before any device
    work: the red-black and bf16 forms exist only for FP32_REFINE."""
    for kw in ({"precision": fs.FS_PRECISION_FP64, "pressure_preconditioner": fs.FS_PRECOND_RED_BLACK},
               {"precision": fs.FS_PRECISION_FP64, "pressure_preconditioner": fs.FS_PRECOND_JACOBI_BF16},
               {"pressure_preconditioner": 9}, {"reliable_delta": 1.5}, {"flux_arithmetic": 3}):
        with pytest.raises(fs.FsError) as e:
            fs.Solver((8, 8, 8), 1.0 / 8, **kw)
        assert e.value.status == fs.FS_INVALID_ARG
