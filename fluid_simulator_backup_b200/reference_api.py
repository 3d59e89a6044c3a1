"""Host mirror of the reference's interface for the timestep path.

Same class names, method names, argument meaning and script keys as the
reference, so code written against it reads the same; the bodies call the
device-resident C ABI.  The reference runs every method on all worker threads
with a barrier after each loop (MULTITHREADING.h); here work happens once, on
thread_id 0 (the reference's BEGIN_HEAD_THREAD_WORK), and calls from other
thread ids return without doing anything.
"""
import numpy as np

from . import (FS_FLAG_CURVATURE_TYPO, FS_FLAG_FAITHFUL_PROJECTION, FS_FLAG_REINIT_TYPO, FS_PRECISION_FP32_REFINE,
               FS_PRECISION_FP64, FS_STOP_ABSOLUTE, FS_STOP_RELATIVE, FS_VELOCITY_ENO3, FS_VELOCITY_WENO5, FsError,
               Solver, default_params, pcg_csr)
from .script import SCRIPT_BLOCK, SCRIPT_READER


class GRID_STRUCTURE_3D:
    """Uniform grid as the reference defines it (GRID_STRUCTURE_3D.h:91-137):
    dx = (max - min)/(res - 1)."""

    def __init__(self, res=(1, 1, 1), start=(0, 0, 0), mn=(0.0, 0.0, 0.0), mx=(1.0, 1.0, 1.0)):
        self.i_res, self.j_res, self.k_res = (int(a) for a in res)
        self.i_start, self.j_start, self.k_start = (int(a) for a in start)
        self.x_min, self.y_min, self.z_min = (float(a) for a in mn)
        self.x_max, self.y_max, self.z_max = (float(a) for a in mx)
        # a one-cell axis (the default-constructed grid) has no spacing of its own
        self.dx = (self.x_max - self.x_min) / max(self.i_res - 1, 1)
        self.dy = (self.y_max - self.y_min) / max(self.j_res - 1, 1)
        self.dz = (self.z_max - self.z_min) / max(self.k_res - 1, 1)

    def InitializeFromBlock(self, block):
        self.__init__(block.GetVector3("base_grid_resolution", (1, 1, 1)), block.GetVector3("start_indices", (0, 0, 0)),
                      block.GetVector3("base_grid_min", (0, 0, 0)), block.GetVector3("base_grid_max", (1, 1, 1)))
        scale = block.GetFloat("resolution_scale", 1.0)
        if scale != 1.0:
            raise ValueError("resolution_scale != 1 is not supported")
        return self


class CSR_MATRIX:
    """CSR system in the reference's layout (CSR_MATRIX.h:10-35)."""

    def __init__(self, values, column_index, row_ptr):
        self.values = np.asarray(values, dtype=np.float64)
        self.column_index = np.asarray(column_index, dtype=np.int32)
        self.row_ptr = np.asarray(row_ptr, dtype=np.int32)
        self.N = len(self.row_ptr) - 1
        self.nz = len(self.values)


class LINEAR_SOLVER:
    """Plugin base class (LINEAR_SOLVER.h:36): Solve is overridden."""

    def __init__(self):
        self.tolerance = 1.0
        self.sqr_tolerance = 1.0
        self.max_iteration = 10
        self.num_iteration = 0
        self.residual = 1e8

    def Initialize(self, multithreading, tolerance, max_iteration):
        self.max_iteration = int(max_iteration)
        self.SetTolerance(tolerance)

    def SetTolerance(self, tolerance):
        self.tolerance = float(tolerance)
        self.sqr_tolerance = self.tolerance ** 2

    def Solve(self, thread_id, A, x, b, bc=None):
        raise NotImplementedError("LINEAR_SOLVER::Solve is virtual")


class CUDA_PCG_METHOD(LINEAR_SOLVER):
    """Jacobi-PCG on the GPU with the reference's stopping test r.z < tol^2
    (PCG_METHOD.cpp:87); `relative=True` stops on ||r||/||b|| instead.
    x (a float64 numpy array) is the initial guess and is overwritten."""

    def __init__(self, relative=False):
        super().__init__()
        self.relative = relative

    def Solve(self, thread_id, A, x, b, bc=None):
        if thread_id != 0:
            return
        out, it, res, status = pcg_csr(A.values, A.column_index, A.row_ptr, b, x, self.tolerance, self.max_iteration,
                                       FS_STOP_RELATIVE if self.relative else FS_STOP_ABSOLUTE)
        x[...] = out
        self.num_iteration = it
        self.residual = res


def velocity_scheme(vel_block):
    """VELOCITY_ADVECTION { use_5th_weno_v, use_3rd_eno_v } (ADVECTION_3D.h:109-112,
    317-328): ENO3 when only use_3rd_eno_v is set, else WENO5.  With both set the
    reference applies WENO5 and then ENO3 to the same fields in one stage; that
    double advection is refused."""
    weno = vel_block.GetBoolean("use_5th_weno_v", False)
    eno = vel_block.GetBoolean("use_3rd_eno_v", False)
    if weno and eno:
        raise ValueError("VELOCITY_ADVECTION selects both use_5th_weno_v and use_3rd_eno_v")
    return FS_VELOCITY_ENO3 if eno else FS_VELOCITY_WENO5


def params_from_block(block, base_grid):
    """fs_params from a FLUID_SOLVER_UNIFORM_AIR_WATER block; keys and
    defaults as EULERIAN_FLUID_SOLVER_3D.h:192-260, ADVECTION_3D and
    PROJECTION_3D.h:178-230 read them.  New keys: precision ("fp64" or
    "fp32_refine"), relative_tolerance, inner_tolerance, max_outer,
    semi_implicit_approach, viscosity_tolerance, corrected_projection."""
    proj = block.FindBlock("PROJECTION_WATER")
    adv = block.FindBlock("LEVELSET_ADVECTION")
    water_drop = proj.GetBoolean("water_drop", False)
    bubble = proj.GetBoolean("air_bubble_rising", False)
    if water_drop == bubble:
        raise ValueError("exactly one of PROJECTION_WATER.water_drop / air_bubble_rising must be true")
    wd, ad = block.GetFloat("water_density", 1.0), block.GetFloat("air_density", 1.0)
    wv, av = block.GetFloat("water_viscosity", 1.0), block.GetFloat("air_viscosity", 0.0)
    neg = (wd, wv) if water_drop else (ad, av)
    pos = (ad, av) if water_drop else (wd, wv)
    precision = block.GetString("precision", "fp64")
    if precision not in ("fp64", "fp32_refine"):
        raise ValueError(f"precision must be fp64 or fp32_refine, got {precision!r}")
    p = default_params(
        rho_neg=neg[0], rho_pos=pos[0], mu_neg=neg[1], mu_pos=pos[1],
        gravity=block.GetVector3("gravity", (0.0, -9.8, 0.0)),
        weno_epsilon=adv.GetFloat("epsilon", 10e-6),
        # EULERIAN_FLUID_SOLVER_3D.h:201-202, 2198-2225: Sussman pseudo-steps only
        # with sussmanstyle_reinitialization, fast sweeping before them with
        # fastsweeping_reinitialization (both default false)
        reinit_iterations=(block.GetInteger("iteration_number_for_reinitialization", 10)
                           if block.GetBoolean("sussmanstyle_reinitialization", False) else 0),
        fast_sweeping=1 if block.GetBoolean("fastsweeping_reinitialization", False) else 0,
        reinit_scaling=block.GetInteger("scaling_number_for_reinitialization", 5),
        order=block.GetInteger("order_for_time_advancing", 1),
        precision=FS_PRECISION_FP32_REFINE if precision == "fp32_refine" else FS_PRECISION_FP64,
        stop=FS_STOP_RELATIVE if proj.GetBoolean("relative_tolerance", False) else FS_STOP_ABSOLUTE,
        tolerance=proj.GetFloat("tolerance", 1e-4),
        max_iteration=proj.GetInteger("max_iteration", 30),
        inner_tolerance=proj.GetFloat("inner_tolerance", 1e-2),
        max_outer=proj.GetInteger("max_outer", 20),
        # semi_implicit_approach = false: the reference's air/water explicit update
        viscosity=1 if block.GetBoolean("semi_implicit_approach", True) else 2,
        viscosity_tolerance=block.GetFloat("viscosity_tolerance", 1e-8),
        flags=0 if block.GetBoolean("corrected_projection", True) else FS_FLAG_FAITHFUL_PROJECTION,
        surface_tension=block.GetFloat("surface_tension", 0.0),
        velocity_scheme=velocity_scheme(block.FindBlock("VELOCITY_ADVECTION")),
        velocity_epsilon=block.FindBlock("VELOCITY_ADVECTION").GetFloat("epsilon", 10e-6),
    )
    if p.precision == FS_PRECISION_FP32_REFINE:
        p.stop = FS_STOP_RELATIVE
    if abs(base_grid.dx - base_grid.dy) > 1e-12 * base_grid.dx or abs(base_grid.dx - base_grid.dz) > 1e-12 * base_grid.dx:
        raise ValueError("the solver needs a uniform grid (dx = dy = dz)")
    return p


def pipe_params_from_script(world, fluid_block, grid):
    """fs_params for the reference's oil/water vertical pipe (pipe = 1) from
    its SIMULATION_WORLD block (a, R2, CFL; SIMULATION_WORLD.h:119-125) and
    FLUID_SOLVER_UNIFORM_OIL_WATER block, with the dimensionless constants
    the reference derives from them (EULERIAN_FLUID_SOLVER_3D.h:496-514):
      R1 = R2/a,  f = g (oil - K water)/(K - 1),
      A = (a^2 - 1) + (m K + 2 (K - 1) ln a),
      V0 = (f + water g) R1^2/(4 water_viscosity) A,
      J = sigma R1 oil/oil_viscosity^2,  Re = oil R1 |V0|/oil_viscosity,
      We = Re^2/J.
    The projection's densities are 1 (oil, phi <= 0) and water/oil; the
    operators run as the reference's do (its Sussman and curvature slips,
    the deflated pressure system, PCG to r.z < tol^2).  The pipe's
    viscosity is not built, so the script must switch the sourcing step off
    (is_sourcing_active = false)."""
    if fluid_block.GetBoolean("is_sourcing_active", True):
        raise ValueError("the pipe mode's viscosity is not built: set is_sourcing_active = false in "
                         "FLUID_SOLVER_UNIFORM_OIL_WATER")
    if not fluid_block.GetBoolean("dimensionless_form", False):
        raise ValueError("the pipe mode is built for dimensionless_form = true")
    if fluid_block.FindBlock("VELOCITY_ADVECTION").GetBoolean("use_5th_weno_v", False):
        raise ValueError("the pipe mode advects the velocity with ENO3 (use_3rd_eno_v) only")
    a, R2 = world.GetFloat("a", 1.0), world.GetFloat("R2", 1.0)
    m, eta = fluid_block.GetFloat("m", 1.0), fluid_block.GetFloat("eta", 1.0)
    K, g = fluid_block.GetFloat("K", 1.0), fluid_block.GetFloat("g", 1.0)
    wd, od = fluid_block.GetFloat("water_density", 1.0), fluid_block.GetFloat("oil_density", 1.0)
    wv, ov = fluid_block.GetFloat("water_viscosity", 1.0), fluid_block.GetFloat("oil_viscosity", 0.0)
    sigma = fluid_block.GetFloat("surface_tension", 0.0)
    R1 = R2 / a
    f = 1.0 / (K - 1.0) * g * (od - K * wd)
    A = (a * a - 1.0) + (m * K + 2.0 * (K - 1) * np.log(a))
    V0 = (f + wd * g) * (R1 * R1) / (4.0 * wv) * A
    J = sigma * R1 * od / (ov * ov)
    Re = (od * R1 * abs(V0)) / ov
    We = (1.0 / J) * (Re * Re)
    proj = fluid_block.FindBlock("PROJECTION_WATER")
    adv = fluid_block.FindBlock("LEVELSET_ADVECTION")
    return default_params(
        pipe=1, pipe_radius=a, grid_min=(grid.x_min, grid.y_min, grid.z_min),
        grid_max=(grid.x_max, grid.y_max, grid.z_max), pipe_R1=R1, pipe_V0=float(V0), pipe_f=f, pipe_eta=eta,
        pipe_oil_density=od, pipe_We=float(We), rho_neg=1.0, rho_pos=wd / od,
        gravity=fluid_block.GetVector3("gravity", (0.0, -9.8, 0.0)),
        weno_epsilon=adv.GetFloat("epsilon", 10e-6),
        reinit_iterations=(fluid_block.GetInteger("iteration_number_for_reinitialization", 10)
                           if fluid_block.GetBoolean("sussmanstyle_reinitialization", False) else 0),
        reinit_scaling=fluid_block.GetInteger("scaling_number_for_reinitialization", 5),
        order=fluid_block.GetInteger("order_for_time_advancing", 1),
        stop=FS_STOP_ABSOLUTE, tolerance=proj.GetFloat("tolerance", 1e-4),
        max_iteration=proj.GetInteger("max_iteration", 30), viscosity=0,
        flags=FS_FLAG_FAITHFUL_PROJECTION | FS_FLAG_REINIT_TYPO | FS_FLAG_CURVATURE_TYPO,
        velocity_scheme=FS_VELOCITY_ENO3, cfl=world.GetFloat("CFL", 0.5))


class PROJECTION_3D:
    """Pressure projection bound to a solver's fields (PROJECTION_3D.h:416)."""

    def __init__(self, solver):
        self._s = solver
        self.last_report = None

    def Solve(self, thread_id, dt):
        if thread_id != 0:
            return
        self.last_report = self._s.project(dt, allow_not_converged=True)

    @property
    def pressure_field(self):
        return self._s.download("pressure")

    @property
    def divergence_field(self):
        return self._s.download("divergence")


class EULERIAN_FLUID_SOLVER_3D:
    """Device-resident replacement of the reference's solver class."""

    def __init__(self):
        self.solver = None
        self.water_projection = None
        self.base_grid = None
        self.order_for_time_advancing = 1
        self.last_report = None

    def InitializeFromScriptBlock(self, multithreading, world_grid, fluid_solver_block):
        self.base_grid = world_grid
        p = params_from_block(fluid_solver_block, world_grid)
        self.order_for_time_advancing = p.order
        self.solver = Solver((world_grid.i_res, world_grid.j_res, world_grid.k_res), world_grid.dx, p)
        self.water_projection = PROJECTION_3D(self.solver)
        return self

    @classmethod
    def FromScript(cls, path, cfl=None):
        """Build from a reference .sim file: the air/water box mode, or the
        oil/water vertical pipe (SIMULATION_WORLD.h:119-122, the mode the
        reference's own four scripts select) with its sourcing step off
        (pipe_params_from_script).  Pipe scripts that need the pipe's
        viscosity, and horizontal pipes, are refused rather than run wrong."""
        r = SCRIPT_READER(path)
        world = r.FindBlock("SIMULATION_WORLD")
        if world.GetBoolean("oil_water_simulation", False):
            disc = world.FindBlock("WORLD_DISCRETIZATION_OIL_WATER")
            if not disc.FindBlock("PIPE_OPTIONS").GetBoolean("is_vertical", False):
                raise ValueError("the pipe mode is built for the vertical pipe (PIPE_OPTIONS.is_vertical) only")
            grid = GRID_STRUCTURE_3D().InitializeFromBlock(disc.FindBlock("GRID_STRUCTURE_3D_VERTICAL"))
            p = pipe_params_from_script(world, r.FindBlock("FLUID_SOLVER_UNIFORM_OIL_WATER"), grid)
            if cfl is not None:
                p.cfl = cfl
            s = cls()
            s.base_grid = grid
            s.order_for_time_advancing = p.order
            s.solver = Solver((grid.i_res, grid.j_res, grid.k_res), grid.dx, p)
            s.water_projection = PROJECTION_3D(s.solver)
            return s
        grid = GRID_STRUCTURE_3D().InitializeFromBlock(
            world.FindBlock("WORLD_DISCRETIZATION_AIR_WATER").FindBlock("GRID_STRUCTURE_3D_LARGE"))
        s = cls().InitializeFromScriptBlock(None, grid, r.FindBlock("FLUID_SOLVER_UNIFORM_AIR_WATER"))
        s.solver.set_params(cfl=cfl if cfl is not None else world.GetFloat("CFL", 0.5))
        return s

    # fields -----------------------------------------------------------------
    @property
    def water_levelset(self):
        return self.solver.download("phi")

    @water_levelset.setter
    def water_levelset(self, a):
        self.solver.upload("phi", a)

    def velocity(self):
        return tuple(self.solver.download(k) for k in "uvw")

    def set_velocity(self, u, v, w):
        for k, a in zip("uvw", (u, v, w)):
            self.solver.upload(k, a)

    # stepping ---------------------------------------------------------------
    def AdvanceOneTimeStepThread(self, thread_id, dt):
        if thread_id != 0:
            return
        self.last_report = self.solver.step(dt, allow_not_converged=True)

    def CFLOneTimeStep(self):
        """dt limit before the CFL factor (the reference multiplies by CFL in
        SIMULATION_WORLD)."""
        return self.solver.cfl_dt() / self.solver.params.cfl

    # level set ----------------------------------------------------------------
    def ReinitializeByFastSweeping(self, thread_id):
        """water_levelset->ReinitializeByFastSweeping (LEVELSET_3D.h:601): the
        solver's sweep direction, which then advances."""
        if thread_id == 0:
            self.solver.fast_sweeping(-1, 1)

    def FullFastSweepingMethodThreaded(self, corrected=False):
        """LEVELSET_3D.h:828-835: four calls in sweep directions 0..3, each
        from its own set-up; corrected: one set-up, then all eight sweeps."""
        if corrected:
            self.solver.fast_sweeping(0, 4)
        else:
            for d in range(4):
                self.solver.fast_sweeping(d, 1)


class WRITE_LEVELSET:
    """WRITE_LEVELSET (WRITE_LEVELSET.h:8-84) over a solver mirror: the water
    level set's surface as an OBJ file named by the caller."""

    def __init__(self, solver):
        self.solver = solver

    def WriteOBJ(self, path):
        self.solver.solver.write_obj(path)


__all__ = ["GRID_STRUCTURE_3D", "CSR_MATRIX", "LINEAR_SOLVER", "CUDA_PCG_METHOD", "PROJECTION_3D",
           "EULERIAN_FLUID_SOLVER_3D", "WRITE_LEVELSET", "params_from_block", "SCRIPT_BLOCK", "SCRIPT_READER", "FsError",
           "FS_PRECISION_FP64"]
