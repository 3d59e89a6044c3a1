"""The reference's oil/water pipe scripts through the host mirror's script
reader (EULERIAN_FLUID_SOLVER_3D.FromScript): the dimensionless constants it
derives must be the reference's own (fixture pipe_frame, made from the
reference's build), and scripts it cannot run are refused.  CPU only: the
reader builds fs_params without touching a GPU."""
import os

import numpy as np
import pytest

from fluid_simulator_backup_b200 import reference_api as R
from fluid_simulator_backup_b200.script import SCRIPT_READER
from oracle import refsim

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def frame_fixture():
    return dict(np.load(os.path.join(GOLD, "pipe_frame.npz")))


def write(tmp_path, g, **kw):
    n = tuple(int(x) for x in g["n"])
    return refsim.write_pipe_sim(str(tmp_path / "pipe.sim"), n, tuple(g["lo"]), tuple(g["hi"]), **kw)


def params(path):
    r = SCRIPT_READER(path)
    world = r.FindBlock("SIMULATION_WORLD")
    disc = world.FindBlock("WORLD_DISCRETIZATION_OIL_WATER")
    grid = R.GRID_STRUCTURE_3D().InitializeFromBlock(disc.FindBlock("GRID_STRUCTURE_3D_VERTICAL"))
    return R.pipe_params_from_script(world, r.FindBlock("FLUID_SOLVER_UNIFORM_OIL_WATER"), grid), grid


def test_pipe_script_gives_the_reference_constants(tmp_path):
    g = frame_fixture()
    p, grid = params(write(tmp_path, g, sourcing=False))
    assert p.pipe == 1 and p.viscosity == 0 and p.order == 2
    assert p.pipe_radius == float(g["a"])
    for mine, ref in ((p.pipe_R1, "R1"), (p.pipe_V0, "V0"), (p.pipe_f, "f"), (p.pipe_eta, "eta"), (p.pipe_We, "We")):
        assert mine == float(g[ref]), ref
    assert p.pipe_oil_density == float(g["oil_density"])
    assert p.rho_neg == 1.0 and p.rho_pos == float(g["water_density"]) / float(g["oil_density"])
    assert tuple(p.grid_min) == tuple(float(x) for x in g["lo"])
    assert tuple(p.grid_max) == tuple(float(x) for x in g["hi"])
    assert abs(grid.dx - (float(g["hi"][0]) - float(g["lo"][0])) / (int(g["n"][0]) - 1)) < 1e-15
    assert p.cfl == float(g["cfl_number"])


def test_pipe_script_needs_the_sourcing_step_off(tmp_path):
    g = frame_fixture()
    with pytest.raises(ValueError, match="is_sourcing_active"):
        params(write(tmp_path, g, sourcing=True))


def test_horizontal_pipe_is_refused(tmp_path):
    g = frame_fixture()
    with pytest.raises(ValueError, match="vertical"):
        R.EULERIAN_FLUID_SOLVER_3D.FromScript(write(tmp_path, g, sourcing=False, vertical=False))
