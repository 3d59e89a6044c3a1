"""ctypes access to the headless reference build (oracle/_ref/libfsref.so).

Test infrastructure only: golden-vector generation, reference-parity checks
and the timed CPU baseline call into the reference solver through this
module; the product path never imports it.

The reference is configured the way its own application is, through a `.sim`
script (SCRIPT_READER block syntax).  `write_sim` emits an air/water box
scenario whose keys are the ones the reference reads:
  SIMULATION_WORLD / WORLD_DISCRETIZATION_AIR_WATER / GRID_STRUCTURE_3D_LARGE
  (SIMULATION_WORLD.h InitializeFormScript, WORLD_DISCRETIZATION_3D.h:73-90),
  FLUID_SOLVER_UNIFORM_AIR_WATER (EULERIAN_FLUID_SOLVER_3D.h:192-260),
  LEVELSET_ADVECTION / VELOCITY_ADVECTION (ADVECTION_3D.h InitializeFromBlock),
  PROJECTION_WATER (PROJECTION_3D.h:178-230).
The grid is n^3 cells on the unit cube: base_grid_min = 0 and
base_grid_max = (n-1)/n so that dx = (max-min)/(res-1) = 1/n
(GRID_STRUCTURE_3D.h:115).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# FSREF_LIB selects another build of the same sources in oracle/_ref/ (the
# timed CPU baseline also tries libfsref_o3.so); goldens use libfsref.so
LIB_PATH = os.path.join(HERE, "_ref", os.environ.get("FSREF_LIB", "libfsref.so"))

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def available():
    return os.path.exists(LIB_PATH)


def _lib():
    lib = ctypes.CDLL(LIB_PATH)
    lib.fsref_create.restype = ctypes.c_void_p
    lib.fsref_create.argtypes = [ctypes.c_char_p]
    lib.fsref_destroy.argtypes = [ctypes.c_void_p]
    lib.fsref_dims.argtypes = [ctypes.c_void_p, _ip]
    lib.fsref_dx.restype = ctypes.c_double
    lib.fsref_dx.argtypes = [ctypes.c_void_p]
    lib.fsref_set.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
    lib.fsref_get.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
    lib.fsref_levelset_ghost.argtypes = [ctypes.c_void_p, _dp]
    lib.fsref_weno5_levelset.argtypes = [ctypes.c_void_p, ctypes.c_double]
    lib.fsref_weno5_velocity.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
    lib.fsref_reinitialization.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
    lib.fsref_projection.restype = ctypes.c_int
    lib.fsref_projection.argtypes = [ctypes.c_void_p, ctypes.c_double]
    lib.fsref_poisson_rows.restype = ctypes.c_int
    lib.fsref_poisson_rows.argtypes = [ctypes.c_void_p]
    lib.fsref_poisson_nnz.restype = ctypes.c_int
    lib.fsref_poisson_nnz.argtypes = [ctypes.c_void_p]
    lib.fsref_poisson_csr.argtypes = [ctypes.c_void_p, _dp, _ip, _ip, _dp, _dp]
    lib.fsref_divergence.argtypes = [ctypes.c_void_p, _dp]
    lib.fsref_viscosity.argtypes = [ctypes.c_void_p, ctypes.c_double]
    lib.fsref_viscosity_ghosted.argtypes = [ctypes.c_void_p, _dp, ctypes.c_double]
    lib.fsref_semi_implicit_solve.restype = ctypes.c_int
    lib.fsref_semi_implicit_solve.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp]
    lib.fsref_cfl.restype = ctypes.c_double
    lib.fsref_cfl.argtypes = [ctypes.c_void_p]
    lib.fsref_curvature.argtypes = [ctypes.c_void_p, _dp]
    lib.fsref_write_levelset.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    lib.fsref_eno3_velocity.argtypes = [ctypes.c_void_p, ctypes.c_double]
    lib.fsref_fast_sweeping.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.fsref_marching_cubes.restype = ctypes.c_int
    lib.fsref_marching_cubes.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int, _ip, ctypes.c_int, _ip]
    lib.fsref_advance_frame.restype = ctypes.c_int
    lib.fsref_advance_frame.argtypes = [ctypes.c_void_p, _dp]
    lib.fsref_set_pressure_tolerance.argtypes = [ctypes.c_void_p, ctypes.c_double]
    lib.fsref_linear_solve.restype = ctypes.c_int
    lib.fsref_linear_solve.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _ip, _ip, _dp, _dp]
    if hasattr(lib, "fsref_pipe_params"):
        lib.fsref_pipe_params.argtypes = [ctypes.c_void_p, _dp]
        lib.fsref_boundary_levelset.argtypes = [ctypes.c_void_p, _dp]
        lib.fsref_ghost_copy.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        lib.fsref_boundary_faces.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        lib.fsref_adv_ghost.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        lib.fsref_fixed.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_ubyte)]
        for fn in ("fsref_pipe_levelset_advection", "fsref_pipe_velocity_advection", "fsref_pipe_reinitialization",
                   "fsref_pipe_gravity"):
            getattr(lib, fn).argtypes = [ctypes.c_void_p, ctypes.c_double]
    if hasattr(lib, "fsref_pipe_viscosity"):
        lib.fsref_pipe_viscosity.argtypes = [ctypes.c_void_p, ctypes.c_double]
        lib.fsref_visc_field.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
    if hasattr(lib, "fsref_pipe_projection"):
        lib.fsref_pipe_projection.restype = ctypes.c_int
        lib.fsref_pipe_projection.argtypes = [ctypes.c_void_p, ctypes.c_double]
        lib.fsref_projection_jc.argtypes = [ctypes.c_void_p, _dp]
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = _lib()
    return _LIB


def write_sim(path, n, *, water_drop=True, threads=1, tolerance=1e-10, max_iteration=100000,
              solver="PCG", reinit_iterations=10, reinit_scaling=5, epsilon=1e-6,
              water_density=1000.0, air_density=1.0, water_viscosity=1e-3, air_viscosity=1.8e-5,
              gravity=(0.0, -9.8, 0.0), order=3, cfl=0.5, velocity_weno=True, surface_tension=0.0,
              fast_sweeping=False, sussman=True):
    """Write an air/water box scenario in the reference's .sim syntax."""
    hi = (n - 1) / n
    b = lambda v: "true" if v else "false"
    # The script's number syntax has no exponent (SCRIPT_READER.cpp:8):
    # every real is written positionally at full double precision.
    r = lambda x: np.format_float_positional(float(x), unique=True, trim="-")
    text = f"""SIMULATION_WORLD
{{
	dt = 0.001
	max_dt = 100
	num_substeps = 1
	CFL = {r(cfl)}
	frame_rate = 30
	use_eulerian_solver = true
	use_sph_solver = false
	use_solid_solver = false
	use_sph_levelset = false
	number_of_threads = {threads}
	use_field_boundary = false
	last_frame = 100000
	auto_run = false
	air_water_simulation = true
	oil_water_simulation = false
	WORLD_DISCRETIZATION_AIR_WATER
	{{
		large_bubble = true
		small_bubble = false
		GRID_STRUCTURE_3D_LARGE
		{{
			resolution_scale = 1
			start_indices = (0,0,0)
			base_grid_resolution = ({n}, {n}, {n})
			base_grid_min = (0, 0, 0)
			base_grid_max = ({r(hi)}, {r(hi)}, {r(hi)})
		}}
		padding_width = 2
	}}
	LOG
	{{
		max_log_level = 1
		use_log_file = false
		display_accum_time = false
		use_log_screen = false
		output_log_file_name = "log.txt"
	}}
}}

FLUID_SOLVER_UNIFORM_AIR_WATER
{{
	use_water_solver = true
	is_Levelset_advection_active = true
	is_Velocity_advection_active = true
	is_external_force_active = true
	is_sourcing_active = true
	is_projection_active = true
	fastsweeping_reinitialization = {b(fast_sweeping)}
	sussmanstyle_reinitialization = {b(sussman)}
	scaling_number_for_reinitialization = {reinit_scaling}
	iteration_number_for_reinitialization = {reinit_iterations}
	use_delta_function_formulation = true
	curvature_by_normal_vector = false
	curvature_by_levelset = true
	CSF_model = false
	order_for_time_advancing = {order}
	LEVELSET_ADVECTION
	{{
		use_csl = false
		use_5th_weno = true
		use_3rd_eno = false
		epsilon = {r(epsilon)}
	}}
	VELOCITY_ADVECTION
	{{
		use_5th_weno_v = {b(velocity_weno)}
		use_3rd_eno_v = {b(not velocity_weno)}
		epsilon = {r(epsilon)}
	}}
	PROJECTION_WATER
	{{
		tolerance = {r(tolerance)}
		max_iteration = {max_iteration}
		air_bubble_rising = {b(not water_drop)}
		water_drop = {b(water_drop)}
		use_previous_pressure = false
		poisson_solver_type = "{solver}"
		use_2nd_order = false
		use_variable_density = true
		Dirichlet_Boundary_Condition = false
		Neumann_Boundary_Condition = true
	}}
	ghost_width = 3
	use_water_levelset = true
	gravity = ({r(gravity[0])}, {r(gravity[1])}, {r(gravity[2])})
	water_viscosity = {r(water_viscosity)}
	water_density = {r(water_density)}
	surface_tension = {r(surface_tension)}
	air_viscosity = {r(air_viscosity)}
	air_density = {r(air_density)}
}}
"""
    with open(path, "w") as f:
        f.write(text)
    return path


def write_pipe_sim(path, res, grid_min, grid_max, *, vertical=True, threads=1, a=1.61, R2=0.47625, A_0=0.1,
                   alpha=2.4, m=0.00166, eta=1.1, K=-2.03030303, g=-980.0, water_density=0.995, oil_density=0.905,
                   water_viscosity=0.01, oil_viscosity=6.01, surface_tension=8.54, gravity=(0.0, -980.0, 0.0),
                   order=2, tolerance=1e-6, max_iteration=10000, reinit_iterations=10, reinit_scaling=2,
                   epsilon=1e-6, periodic_num=5, cfl=0.8, sourcing=True):
    """Write an oil/water pipe scenario in the reference's .sim syntax, with
    the keys of the reference's own pipe scripts (3D_script_1.sim):
    SIMULATION_WORLD (a, R2, A_0, alpha; SIMULATION_WORLD.h:120-129),
    WORLD_DISCRETIZATION_OIL_WATER with PIPE_OPTIONS and the vertical or
    parallel grid (WORLD_DISCRETIZATION_3D.h:91-107),
    FLUID_SOLVER_UNIFORM_OIL_WATER (dimensionless form, m, eta, K, g;
    EULERIAN_FLUID_SOLVER_3D.h:192-560) and an OBJECT_LIST whose WATER object
    makes the reference seed the core-annular level set and the cylinder's
    boundary level set (SIMULATION_WORLD.cpp:130-300)."""
    b = lambda v: "true" if v else "false"
    r = lambda x: np.format_float_positional(float(x), unique=True, trim="-")
    v3 = lambda t: f"({r(t[0])}, {r(t[1])}, {r(t[2])})"
    grid = f"""
		{{
			resolution_scale = 1
			start_indices = (0,0,0)
			base_grid_resolution = ({res[0]}, {res[1]}, {res[2]})
			base_grid_min = {v3(grid_min)}
			base_grid_max = {v3(grid_max)}
		}}"""
    text = f"""SIMULATION_WORLD
{{
	dt = 0.00001
	max_dt = 1000000
	num_substeps = 1
	CFL = {r(cfl)}
	frame_rate = 30
	use_eulerian_solver = true
	use_sph_solver = false
	use_solid_solver = false
	use_sph_levelset = false
	number_of_threads = {threads}
	use_field_boundary = false
	last_frame = 100000
	auto_run = false
	air_water_simulation = false
	oil_water_simulation = true
	a = {r(a)}
	R2 = {r(R2)}
	A_0 = {r(A_0)}
	alpha = {r(alpha)}
	WORLD_DISCRETIZATION_OIL_WATER
	{{
		PIPE_OPTIONS
		{{
			is_vertical = {b(vertical)}
			is_parallel = {b(not vertical)}
		}}
		GRID_STRUCTURE_3D_VERTICAL{grid}
		GRID_STRUCTURE_3D_PARALLEL{grid}
		padding_width = 2
	}}
	LOG
	{{
		max_log_level = 1
		use_log_file = false
		display_accum_time = false
		use_log_screen = false
		output_log_file_name = "log.txt"
	}}
}}

FLUID_SOLVER_UNIFORM_OIL_WATER
{{
	use_water_solver = true
	is_Levelset_advection_active = true
	is_Velocity_advection_active = true
	is_external_force_active = true
	is_sourcing_active = {b(sourcing)}
	is_projection_active = true
	fastsweeping_reinitialization = false
	sussmanstyle_reinitialization = true
	scaling_number_for_reinitialization = {reinit_scaling}
	iteration_number_for_reinitialization = {reinit_iterations}
	use_delta_function_formulation = true
	curvature_by_normal_vector = false
	curvature_by_levelset = true
	order_for_time_advancing = {order}
	semi_implicit_approach = true
	dimensionless_form = true
	CSF_model = false
	is_periodic = true
	periodic_num = {periodic_num}
	m = {r(m)}
	eta = {r(eta)}
	K = {r(K)}
	g = {r(g)}
	LEVELSET_ADVECTION
	{{
		use_csl = false
		use_5th_weno = true
		use_3rd_eno = false
		epsilon = {r(epsilon)}
	}}
	VELOCITY_ADVECTION
	{{
		use_5th_weno_v = false
		use_3rd_eno_v = true
		epsilon = {r(epsilon)}
	}}
	PROJECTION_WATER
	{{
		tolerance = {r(tolerance)}
		max_iteration = {max_iteration}
		use_previous_pressure = true
		poisson_solver_type = "PCG"
		use_2nd_order = false
		use_variable_density = true
		Dirichlet_Boundary_Condition = false
		Neumann_Boundary_Condition = true
		regular_boundary = false
		cylindrical_boundary = true
	}}
	ghost_width = 3
	use_water_levelset = true
	gravity = {v3(gravity)}
	water_viscosity = {r(water_viscosity)}
	water_density = {r(water_density)}
	surface_tension = {r(surface_tension)}
	oil_density = {r(oil_density)}
	oil_viscosity = {r(oil_viscosity)}
}}

OBJECT_LIST
{{
	WATER
	{{
		object_type = "FLUID"
		shape_type = "WATER"
		use_sea_surface = false
		use_sphere_bubble = false
		user_defined = false
	}}
}}
"""
    with open(path, "w") as f:
        f.write(text)
    return path


PIPE_PARAMS = ("a", "R1", "m", "eta", "K", "g", "f", "A", "V0", "J", "Re", "We", "water_density", "oil_density",
               "water_viscosity", "oil_viscosity", "surface_tension", "is_vertical", "is_parallel", "x_min", "y_min",
               "z_min", "dx", "dy", "dz")


def _ptr(a, ct=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(ct))


class RefCase:
    """One reference solver instance built from a generated script."""

    FIELDS = {"phi": 0, "u": 1, "v": 2, "w": 3, "p": 4}

    def __init__(self, sim_path):
        self._lib = lib()
        devnull = os.open(os.devnull, os.O_WRONLY)
        saved = os.dup(1)
        os.dup2(devnull, 1)  # the reference prints its configuration on stdout
        try:
            self.h = self._lib.fsref_create(sim_path.encode())
        finally:
            os.dup2(saved, 1)
            os.close(saved)
            os.close(devnull)
        d = (ctypes.c_int * 3)()
        self._lib.fsref_dims(self.h, d)
        self.n = tuple(d)  # (nx, ny, nz)
        self.dx = self._lib.fsref_dx(self.h)

    def close(self):
        if self.h:
            self._lib.fsref_destroy(self.h)
            self.h = None

    def shape(self, name):
        nx, ny, nz = self.n
        return {"phi": (nz, ny, nx), "p": (nz, ny, nx), "u": (nz, ny, nx + 1),
                "v": (nz, ny + 1, nx), "w": (nz + 1, ny, nx)}[name]

    def set(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.shape == self.shape(name), (name, a.shape)
        self._lib.fsref_set(self.h, self.FIELDS[name], _ptr(a))

    def get(self, name):
        a = np.empty(self.shape(name), dtype=np.float64)
        self._lib.fsref_get(self.h, self.FIELDS[name], _ptr(a))
        return a

    def _quiet(self, fn, *args):
        devnull = os.open(os.devnull, os.O_WRONLY)
        saved = os.dup(1)
        os.dup2(devnull, 1)
        try:
            return fn(*args)
        finally:
            os.dup2(saved, 1)
            os.close(saved)
            os.close(devnull)

    def levelset_ghost(self):
        nx, ny, nz = self.n
        a = np.empty((nz + 6, ny + 6, nx + 6))
        self._lib.fsref_levelset_ghost(self.h, _ptr(a))
        return a

    def weno5_levelset(self, dt):
        self._lib.fsref_weno5_levelset(self.h, dt)

    def weno5_velocity(self, dt, own_ghost):
        self._lib.fsref_weno5_velocity(self.h, dt, int(own_ghost))

    def reinitialization(self, dt, refresh_ghosts):
        self._lib.fsref_reinitialization(self.h, dt, int(refresh_ghosts))

    def projection(self, dt):
        return self._quiet(self._lib.fsref_projection, self.h, dt)

    def poisson_csr(self):
        rows = self._lib.fsref_poisson_rows(self.h)
        nnz = self._lib.fsref_poisson_nnz(self.h)
        vals = np.empty(nnz)
        cols = np.empty(nnz, dtype=np.int32)
        rowptr = np.empty(rows + 1, dtype=np.int32)
        b = np.empty(rows)
        x = np.empty(rows)
        self._lib.fsref_poisson_csr(self.h, _ptr(vals), _ptr(cols, ctypes.c_int), _ptr(rowptr, ctypes.c_int), _ptr(b), _ptr(x))
        return vals, cols, rowptr, b, x

    def divergence(self):
        a = np.empty(self.shape("phi"))
        self._lib.fsref_divergence(self.h, _ptr(a))
        return a

    def viscosity(self, dt):
        self._lib.fsref_viscosity(self.h, dt)

    def viscosity_ghosted(self, phi_ghosted, dt):
        """VISCOSITY_3D::ApplyViscosity (air/water, explicit, in place) with
        the level set's first ghost layer from phi_ghosted [(nz+2, ny+2,
        nx+2)] and zero velocity ghosts."""
        a = np.ascontiguousarray(phi_ghosted, dtype=np.float64)
        nx, ny, nz = self.n
        assert a.shape == (nz + 2, ny + 2, nx + 2)
        self._lib.fsref_viscosity_ghosted(self.h, _ptr(a), float(dt))

    def semi_implicit_solve(self, comp, coef, explicit_term):
        name = {1: "u", 2: "v", 3: "w"}[comp]
        coef = np.ascontiguousarray(coef, dtype=np.float64)
        ex = np.ascontiguousarray(explicit_term, dtype=np.float64)
        out = np.empty(self.shape(name))
        it = self._quiet(self._lib.fsref_semi_implicit_solve, self.h, comp, _ptr(coef), _ptr(ex), _ptr(out))
        return out, it

    def cfl(self):
        return self._lib.fsref_cfl(self.h)

    def eno3_velocity(self, dt):
        return self._quiet(self._lib.fsref_eno3_velocity, self.h, dt)

    def fast_sweeping(self, direction):
        """LEVELSET_3D::ReinitializeByFastSweeping (without its Update) with
        sweep_direction = direction, on the injected level set."""
        return self._quiet(self._lib.fsref_fast_sweeping, self.h, int(direction))

    def marching_cubes(self, cap=200000):
        """WRITE_LEVELSET::WriteOBJ's surface of the injected level set:
        (vertices [nv, 3], vertex normals [nv, 3], triangles [nt, 3] of 1-based
        vertex indices)."""
        xyz = np.zeros((cap, 3)); nrm = np.zeros((cap, 3)); tri = np.zeros((cap, 3), np.int32)
        nt = ctypes.c_int()
        nv = self._quiet(self._lib.fsref_marching_cubes, self.h, _ptr(xyz), _ptr(nrm), cap, _ptr(tri, ctypes.c_int),
                         cap, ctypes.byref(nt))
        if nv > cap or nt.value > cap:
            raise ValueError("surface larger than the buffers")
        return xyz[:nv].copy(), nrm[:nv].copy(), tri[:nt.value].copy()

    def write_levelset(self, path):
        """LEVELSET_3D::Write of the current level set to `path`."""
        self._lib.fsref_write_levelset(self.h, path.encode())

    def curvature(self):
        a = np.empty(self.shape("phi"))
        self._lib.fsref_curvature(self.h, _ptr(a))
        return a

    def advance_frame(self):
        """SIMULATION_WORLD::AdvanceOneFrame: one whole reference timestep
        with dt from its CFL condition.  Returns (dt, PCG iterations of the
        frame's last pressure solve)."""
        dt = ctypes.c_double()
        it = self._quiet(self._lib.fsref_advance_frame, self.h, ctypes.byref(dt))
        return dt.value, it

    def set_pressure_tolerance(self, tol):
        """The PCG stops when r.z < tol^2 (PCG_METHOD.cpp:87)."""
        self._lib.fsref_set_pressure_tolerance(self.h, float(tol))

    def linear_solve(self, vals, cols, rowptr, b, x0):
        n = len(b)
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        cols = np.ascontiguousarray(cols, dtype=np.int32)
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.array(x0, dtype=np.float64)
        it = self._quiet(self._lib.fsref_linear_solve, self.h, n, len(vals), _ptr(vals), _ptr(cols, ctypes.c_int),
                         _ptr(rowptr, ctypes.c_int), _ptr(b), _ptr(x))
        return x, it

    # ---- oil/water pipe mode
    def pipe_params(self):
        out = np.zeros(len(PIPE_PARAMS))
        self._lib.fsref_pipe_params(self.h, _ptr(out))
        return dict(zip(PIPE_PARAMS, out.tolist()))

    def boundary_levelset(self):
        a = np.empty(self.shape("phi"))
        self._lib.fsref_boundary_levelset(self.h, _ptr(a))
        return a

    def ghost_copy(self, name):
        """The ghosted copy (three ghost layers) the operators read: "phi" or a
        velocity component."""
        sh = tuple(d + 6 for d in self.shape(name))
        a = np.empty(sh)
        self._lib.fsref_ghost_copy(self.h, {"phi": 0, "u": 1, "v": 2, "w": 3}[name], _ptr(a))
        return a

    def fixed(self, name):
        a = np.empty(self.shape(name), dtype=np.uint8)
        self._lib.fsref_fixed(self.h, {"u": 0, "v": 1, "w": 2}[name], _ptr(a, ctypes.c_ubyte))
        return a.astype(bool)

    def pipe_levelset_advection(self, dt):
        self._quiet(self._lib.fsref_pipe_levelset_advection, self.h, dt)

    def pipe_velocity_advection(self, dt):
        self._quiet(self._lib.fsref_pipe_velocity_advection, self.h, dt)

    def pipe_reinitialization(self, dt):
        self._quiet(self._lib.fsref_pipe_reinitialization, self.h, dt)

    def pipe_gravity(self, dt):
        self._quiet(self._lib.fsref_pipe_gravity, self.h, dt)

    def pipe_viscosity(self, dt):
        """VISCOSITY_3D::ApplyViscosity of the pipe (semi-implicit, in place)."""
        self._quiet(self._lib.fsref_pipe_viscosity, self.h, dt)

    def visc_field(self, comp, q):
        """The explicit term (q = 0) or coef_q (1..6) of component comp
        ("u", "v", "w") of the last semi-implicit viscosity."""
        a = np.empty(self.shape(comp))
        self._lib.fsref_visc_field(self.h, 7 * "uvw".index(comp) + q, _ptr(a))
        return a

    def pipe_projection(self, dt):
        """EULERIAN_FLUID_SOLVER_3D::Projection of the pipe; returns the PCG
        iteration count."""
        return self._quiet(self._lib.fsref_pipe_projection, self.h, dt)

    def projection_jc(self):
        a = np.empty(self.shape("phi"))
        self._lib.fsref_projection_jc(self.h, _ptr(a))
        return a

    def boundary_faces(self, name):
        """The pipe's boundary level set on the faces of a component, as the
        last velocity set-up computed it."""
        a = np.empty(self.shape(name))
        self._lib.fsref_boundary_faces(self.h, {"u": 0, "v": 1, "w": 2}[name], _ptr(a))
        return a

    def advection_ghost(self, comp, axis):
        """The advection's per-axis ghost copy of component comp ("u", "v",
        "w") read along axis ("x", "y", "z"), with its three ghost layers."""
        sh = tuple(d + 6 for d in self.shape(comp))
        a = np.empty(sh)
        self._lib.fsref_adv_ghost(self.h, 3 * "uvw".index(comp) + "xyz".index(axis), _ptr(a))
        return a
