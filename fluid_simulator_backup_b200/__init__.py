"""B200-native (sm_100a) timestep of the two-phase level-set Navier-Stokes
solver of ByungJoonLee/Fluid_Simulator_BackUp.

The compute path is the in-tree CUDA library ``libfluidb200.so`` (C ABI in
``include/fluid_b200.h``); this package is its Python binding plus a mirror of
the reference's host interface for this path:

  ``EULERIAN_FLUID_SOLVER_3D``  InitializeFromScriptBlock / AdvanceOneTimeStepThread
                                / CFLOneTimeStep (EULERIAN_FLUID_SOLVER_3D.h:192,803,2673)
  ``PROJECTION_3D``             Solve(thread_id, dt) (PROJECTION_3D.h:416)
  ``CUDA_PCG_METHOD``           LINEAR_SOLVER::Solve(thread_id, A, x, b, bc) (LINEAR_SOLVER.h:36)
  ``SCRIPT_READER``             the .sim block reader (SCRIPT_READER.h:161-173)

There is no CPU fallback: importing the package without the built library,
or using it without a CUDA device, raises.
"""
import ctypes
import os

import numpy as np

from .script import SCRIPT_BLOCK, SCRIPT_READER  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfluidb200.so")

FS_OK, FS_INVALID_ARG, FS_OOM, FS_NOT_CONVERGED, FS_NONFINITE, FS_CUDA_ERROR, FS_TIMEOUT, FS_NOT_SUPPORTED = range(8)
FIELD = {"phi": 0, "u": 1, "v": 2, "w": 3, "pressure": 4, "p": 4, "divergence": 5,
         "adj_phi": 6, "adj_u": 7, "adj_v": 8, "adj_w": 9, "curvature": 10}
FS_PRECISION_FP64, FS_PRECISION_FP32_REFINE = 0, 1
FS_STOP_RELATIVE, FS_STOP_ABSOLUTE = 0, 1
FS_FLAG_FAITHFUL_PROJECTION, FS_FLAG_REINIT_TYPO, FS_FLAG_LEVELSET_FORWARD_EULER, FS_FLAG_CURVATURE_TYPO = 1, 2, 4, 8
FS_FLAG_SORT_TYPO, FS_FLAG_VISCOSITY_IN_PLACE = 16, 32
FS_VISCOSITY_OFF, FS_VISCOSITY_SEMI_IMPLICIT, FS_VISCOSITY_EXPLICIT = 0, 1, 2
FS_VELOCITY_WENO5, FS_VELOCITY_ENO3 = 0, 1
FS_PRECOND_DEFAULT, FS_PRECOND_JACOBI, FS_PRECOND_JACOBI_BF16, FS_PRECOND_RED_BLACK = 0, 1, 2, 3
FS_PRECOND_RED_BLACK_JACOBI = 4

EXPORTED = ("fs_params_default", "fs_status_str", "fs_last_error", "fs_create", "fs_destroy", "fs_set_params",
            "fs_memory_bytes", "fs_upload", "fs_download", "fs_upload_device", "fs_download_device", "fs_step",
            "fs_cfl_dt", "fs_project", "fs_advect_levelset", "fs_advect_velocity", "fs_reinitialize", "fs_apply_gravity",
            "fs_viscosity", "fs_pcg_csr", "fs_pcg_csr_noalloc", "fs_adjoint_reset", "fs_adjoint_density_bars",
            "fs_step_adjoint", "fs_advect_levelset_adjoint", "fs_advect_velocity_adjoint", "fs_reinitialize_adjoint",
            "fs_viscosity_adjoint", "fs_project_adjoint", "fs_curvature", "fs_write_levelset", "fs_read_levelset",
            "fs_write_state", "fs_read_state", "fs_fast_sweeping", "fs_surface", "fs_surface_download",
            "fs_write_obj")


class FsError(RuntimeError):
    def __init__(self, status, where, detail=""):
        self.status = status
        super().__init__(f"{where}: {status_str(status)} ({status}){': ' + detail if detail else ''}")


class GridDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("dx", ctypes.c_double)]


class Params(ctypes.Structure):
    _fields_ = [("rho_neg", ctypes.c_double), ("rho_pos", ctypes.c_double), ("mu_neg", ctypes.c_double),
                ("mu_pos", ctypes.c_double), ("gravity", ctypes.c_double * 3), ("weno_epsilon", ctypes.c_double),
                ("reinit_iterations", ctypes.c_int), ("reinit_scaling", ctypes.c_int), ("order", ctypes.c_int),
                ("precision", ctypes.c_int), ("stop", ctypes.c_int), ("tolerance", ctypes.c_double),
                ("max_iteration", ctypes.c_int), ("inner_tolerance", ctypes.c_double), ("max_outer", ctypes.c_int),
                ("viscosity", ctypes.c_int), ("viscosity_tolerance", ctypes.c_double),
                ("viscosity_max_iteration", ctypes.c_int), ("cfl", ctypes.c_double), ("flags", ctypes.c_int),
                ("surface_tension", ctypes.c_double), ("velocity_scheme", ctypes.c_int),
                ("velocity_epsilon", ctypes.c_double), ("fast_sweeping", ctypes.c_int),
                ("pressure_preconditioner", ctypes.c_int), ("reliable_delta", ctypes.c_double),
                ("flux_arithmetic", ctypes.c_int), ("verbose", ctypes.c_int),
                ("host_loop", ctypes.c_int),
                # oil/water vertical pipe mode (0: the box)
                ("pipe", ctypes.c_int), ("pipe_radius", ctypes.c_double), ("grid_min", ctypes.c_double * 3),
                ("grid_max", ctypes.c_double * 3), ("pipe_R1", ctypes.c_double), ("pipe_V0", ctypes.c_double),
                ("pipe_f", ctypes.c_double), ("pipe_eta", ctypes.c_double), ("pipe_oil_density", ctypes.c_double),
                ("pipe_We", ctypes.c_double)]

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if name in ("gravity", "grid_min", "grid_max") else v
        return d


class SolveReport(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("outer_iterations", ctypes.c_int), ("rel_residual", ctypes.c_double),
                ("rz", ctypes.c_double), ("div_l2", ctypes.c_double), ("div_linf", ctypes.c_double),
                ("ms", ctypes.c_float)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class StepReport(ctypes.Structure):
    _fields_ = [("pcg_iterations", ctypes.c_int), ("outer_iterations", ctypes.c_int),
                ("viscosity_iterations", ctypes.c_int), ("projections", ctypes.c_int),
                ("max_rel_residual", ctypes.c_double), ("div_l2", ctypes.c_double), ("div_linf", ctypes.c_double),
                ("ms", ctypes.c_float), ("pcg_ms", ctypes.c_float), ("pcg_launched_iterations", ctypes.c_int),
                ("kernel_launches", ctypes.c_int64)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


_LIB = None


def lib():
    """The loaded CUDA library (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m fluid_simulator_backup_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp, dp, ip, i64p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), \
            ctypes.POINTER(ctypes.c_int64)
        L.fs_params_default.argtypes = [ctypes.POINTER(Params)]
        L.fs_params_default.restype = None
        L.fs_status_str.argtypes = [ctypes.c_int]
        L.fs_status_str.restype = ctypes.c_char_p
        L.fs_last_error.argtypes = []
        L.fs_last_error.restype = ctypes.c_char_p
        L.fs_create.argtypes = [ctypes.POINTER(GridDesc), ctypes.POINTER(Params), ctypes.POINTER(vp)]
        L.fs_destroy.argtypes = [vp]
        L.fs_set_params.argtypes = [vp, ctypes.POINTER(Params)]
        L.fs_memory_bytes.argtypes = [vp, i64p]
        L.fs_upload.argtypes = [vp, ctypes.c_int, vp, vp]
        L.fs_download.argtypes = [vp, ctypes.c_int, vp, vp]
        L.fs_upload_device.argtypes = [vp, ctypes.c_int, vp]
        L.fs_download_device.argtypes = [vp, ctypes.c_int, vp]
        L.fs_step.argtypes = [vp, ctypes.c_double, ctypes.POINTER(StepReport)]
        L.fs_cfl_dt.argtypes = [vp, dp]
        L.fs_project.argtypes = [vp, ctypes.c_double, ctypes.POINTER(SolveReport)]
        L.fs_advect_levelset.argtypes = [vp, ctypes.c_double]
        L.fs_advect_velocity.argtypes = [vp, ctypes.c_double]
        L.fs_reinitialize.argtypes = [vp]
        L.fs_apply_gravity.argtypes = [vp, ctypes.c_double]
        L.fs_fast_sweeping.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.fs_surface.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
        L.fs_surface_download.argtypes = [vp, vp, vp, vp]
        L.fs_write_obj.argtypes = [vp, ctypes.c_char_p]
        L.fs_viscosity.argtypes = [vp, ctypes.c_double, ip]
        L.fs_pcg_csr.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_double, ctypes.c_int,
                                 ctypes.c_int, ip, dp]
        L.fs_pcg_csr_noalloc.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_int, vp, ip, dp]
        L.fs_curvature.argtypes = [vp, dp]
        L.fs_write_levelset.argtypes = [vp, ctypes.c_char_p, dp]
        L.fs_read_levelset.argtypes = [vp, ctypes.c_char_p, dp]
        L.fs_write_state.argtypes = [vp, ctypes.c_char_p]
        L.fs_read_state.argtypes = [vp, ctypes.c_char_p]
        L.fs_adjoint_reset.argtypes = [vp]
        L.fs_adjoint_density_bars.argtypes = [vp, dp, dp]
        L.fs_step_adjoint.argtypes = [vp, ctypes.c_double, ctypes.POINTER(StepReport)]
        L.fs_advect_levelset_adjoint.argtypes = [vp, ctypes.c_double]
        L.fs_advect_velocity_adjoint.argtypes = [vp, ctypes.c_double]
        L.fs_reinitialize_adjoint.argtypes = [vp]
        L.fs_viscosity_adjoint.argtypes = [vp, ctypes.c_double]
        L.fs_project_adjoint.argtypes = [vp, ctypes.c_double]
        for name in EXPORTED:
            if name not in ("fs_params_default", "fs_status_str", "fs_last_error"):
                getattr(L, name).restype = ctypes.c_int
        _LIB = L
    return _LIB


def status_str(s):
    return lib().fs_status_str(int(s)).decode()


def last_error():
    return lib().fs_last_error().decode()


def _check(status, where, allow=()):
    if status != FS_OK and status not in allow:
        raise FsError(status, where, last_error())
    return status


def default_params(**overrides):
    p = Params()
    lib().fs_params_default(ctypes.byref(p))
    for k, v in overrides.items():
        if k in ("gravity", "grid_min", "grid_max"):
            for a in range(3):
                getattr(p, k)[a] = float(v[a])
        else:
            setattr(p, k, v)
    return p


def field_shape(n, name):
    nx, ny, nz = n
    if name.startswith("adj_"):
        name = name[4:]
    return {"phi": (nz, ny, nx), "pressure": (nz, ny, nx), "p": (nz, ny, nx), "divergence": (nz, ny, nx),
            "curvature": (nz, ny, nx), "u": (nz, ny, nx + 1), "v": (nz, ny + 1, nx), "w": (nz + 1, ny, nx)}[name]


class Solver:
    """One device-resident simulation (an fs_ctx)."""

    def __init__(self, n, dx, params=None, **overrides):
        if isinstance(n, int):
            n = (n, n, n)
        self.n = tuple(int(a) for a in n)
        self.dx = float(dx)
        self.params = params if params is not None else default_params(**overrides)
        if params is not None and overrides:
            for k, v in overrides.items():
                setattr(self.params, k, v)
        g = GridDesc(self.n[0], self.n[1], self.n[2], self.dx)
        h = ctypes.c_void_p()
        _check(lib().fs_create(ctypes.byref(g), ctypes.byref(self.params), ctypes.byref(h)), "fs_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().fs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_params(self, **kw):
        for k, v in kw.items():
            if k == "gravity":
                for a in range(3):
                    self.params.gravity[a] = float(v[a])
            else:
                setattr(self.params, k, v)
        _check(lib().fs_set_params(self._h, ctypes.byref(self.params)), "fs_set_params")

    def memory_bytes(self):
        b = ctypes.c_int64()
        _check(lib().fs_memory_bytes(self._h, ctypes.byref(b)), "fs_memory_bytes")
        return b.value

    def shape(self, name):
        return field_shape(self.n, name)

    def upload(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != self.shape(name):
            raise ValueError(f"{name}: expected shape {self.shape(name)}, got {a.shape}")
        _check(lib().fs_upload(self._h, FIELD[name], a.ctypes.data, None), f"fs_upload({name})")

    def download(self, name):
        a = np.empty(self.shape(name), dtype=np.float64)
        _check(lib().fs_download(self._h, FIELD[name], a.ctypes.data, None), f"fs_download({name})")
        return a

    def upload_ptr(self, name, host_ptr):
        """Upload from a raw host pointer to packed FP64 values (e.g. pinned memory)."""
        _check(lib().fs_upload(self._h, FIELD[name], host_ptr, None), f"fs_upload({name})")

    def download_ptr(self, name, host_ptr):
        _check(lib().fs_download(self._h, FIELD[name], host_ptr, None), f"fs_download({name})")

    def upload_device(self, name, dev_ptr):
        _check(lib().fs_upload_device(self._h, FIELD[name], dev_ptr), f"fs_upload_device({name})")

    def download_device(self, name, dev_ptr):
        _check(lib().fs_download_device(self._h, FIELD[name], dev_ptr), f"fs_download_device({name})")

    def step(self, dt, allow_not_converged=False):
        r = StepReport()
        s = lib().fs_step(self._h, float(dt), ctypes.byref(r))
        _check(s, "fs_step", (FS_NOT_CONVERGED,) if allow_not_converged else ())
        out = r.as_dict()
        out["status"] = s
        return out

    def cfl_dt(self):
        d = ctypes.c_double()
        _check(lib().fs_cfl_dt(self._h, ctypes.byref(d)), "fs_cfl_dt")
        return d.value

    def project(self, dt, allow_not_converged=False):
        r = SolveReport()
        s = lib().fs_project(self._h, float(dt), ctypes.byref(r))
        _check(s, "fs_project", (FS_NOT_CONVERGED,) if allow_not_converged else ())
        out = r.as_dict()
        out["status"] = s
        return out

    def advect_levelset(self, dt):
        _check(lib().fs_advect_levelset(self._h, float(dt)), "fs_advect_levelset")

    def advect_velocity(self, dt):
        _check(lib().fs_advect_velocity(self._h, float(dt)), "fs_advect_velocity")

    def apply_gravity(self, dt):
        """EULERIAN_FLUID_SOLVER_3D::ApplyGravity: gravity in the box, the
        dimensionless body force in pipe mode."""
        _check(lib().fs_apply_gravity(self._h, float(dt)), "fs_apply_gravity")

    def reinitialize(self):
        _check(lib().fs_reinitialize(self._h), "fs_reinitialize")

    def surface(self):
        """The zero level set as a closed triangle mesh (marching cubes):
        vertices [nv, 3] (x, y, z), vertex normals [nv, 3], triangles
        [nt, 3] of 1-based vertex numbers."""
        nv, nt = ctypes.c_int64(), ctypes.c_int64()
        _check(lib().fs_surface(self._h, ctypes.byref(nv), ctypes.byref(nt)), "fs_surface")
        xyz = np.empty((nv.value, 3))
        nrm = np.empty((nv.value, 3))
        tri = np.empty((nt.value, 3), dtype=np.int32)
        _check(lib().fs_surface_download(self._h, xyz.ctypes.data, nrm.ctypes.data, tri.ctypes.data),
               "fs_surface_download")
        return xyz, nrm, tri

    def write_obj(self, path):
        """The surface as a Wavefront OBJ file (WRITE_LEVELSET::WriteOBJ)."""
        _check(lib().fs_write_obj(self._h, os.fsencode(path)), "fs_write_obj")

    def fast_sweeping(self, direction=-1, pairs=1):
        """LEVELSET_3D::ReinitializeByFastSweeping on phi (direction -1: the
        context's sweep counter, which advances)."""
        _check(lib().fs_fast_sweeping(self._h, int(direction), int(pairs)), "fs_fast_sweeping")

    def viscosity(self, dt):
        it = ctypes.c_int()
        _check(lib().fs_viscosity(self._h, float(dt), ctypes.byref(it)), "fs_viscosity")
        return it.value

    def write_levelset(self, path, grid_min=(0.0, 0.0, 0.0)):
        """The level set in the reference's LEVELSET_3D binary format."""
        mn = (ctypes.c_double * 3)(*grid_min)
        _check(lib().fs_write_levelset(self._h, str(path).encode(), mn), "fs_write_levelset")

    def read_levelset(self, path):
        """Load a LEVELSET_3D file; returns the grid minimum it records."""
        mn = (ctypes.c_double * 3)()
        _check(lib().fs_read_levelset(self._h, str(path).encode(), mn), "fs_read_levelset")
        return tuple(mn)

    def write_state(self, path):
        _check(lib().fs_write_state(self._h, str(path).encode()), "fs_write_state")

    def read_state(self, path):
        _check(lib().fs_read_state(self._h, str(path).encode()), "fs_read_state")

    def curvature(self):
        """Mean curvature of the current level set and max |kappa| over |phi| < 0.1."""
        m = ctypes.c_double()
        _check(lib().fs_curvature(self._h, ctypes.byref(m)), "fs_curvature")
        return self.download("curvature"), m.value

    # ---- adjoints (FP64 contexts): bars live in the adj_* fields
    def adjoint_reset(self):
        _check(lib().fs_adjoint_reset(self._h), "fs_adjoint_reset")

    def density_bars(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(lib().fs_adjoint_density_bars(self._h, ctypes.byref(a), ctypes.byref(b)), "fs_adjoint_density_bars")
        return a.value, b.value

    def step_adjoint(self, dt, allow_not_converged=False):
        r = StepReport()
        s = lib().fs_step_adjoint(self._h, float(dt), ctypes.byref(r))
        _check(s, "fs_step_adjoint", (FS_NOT_CONVERGED,) if allow_not_converged else ())
        out = r.as_dict()
        out["status"] = s
        return out

    def advect_levelset_adjoint(self, dt):
        _check(lib().fs_advect_levelset_adjoint(self._h, float(dt)), "fs_advect_levelset_adjoint")

    def advect_velocity_adjoint(self, dt):
        _check(lib().fs_advect_velocity_adjoint(self._h, float(dt)), "fs_advect_velocity_adjoint")

    def reinitialize_adjoint(self):
        _check(lib().fs_reinitialize_adjoint(self._h), "fs_reinitialize_adjoint")

    def viscosity_adjoint(self, dt):
        _check(lib().fs_viscosity_adjoint(self._h, float(dt)), "fs_viscosity_adjoint")

    def project_adjoint(self, dt):
        _check(lib().fs_project_adjoint(self._h, float(dt)), "fs_project_adjoint", (FS_NOT_CONVERGED,))


def pcg_csr(values, column_index, row_ptr, b, x0, tolerance, max_iteration, stop=FS_STOP_ABSOLUTE, solver=None):
    """Jacobi-PCG on a CSR system through the C ABI (LINEAR_SOLVER plugin)."""
    vals = np.ascontiguousarray(values, dtype=np.float64)
    cols = np.ascontiguousarray(column_index, dtype=np.int32)
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    bb = np.ascontiguousarray(b, dtype=np.float64)
    x = np.array(x0, dtype=np.float64)
    it = ctypes.c_int()
    res = ctypes.c_double()
    s = lib().fs_pcg_csr(solver.handle if solver else None, len(bb), len(vals), vals.ctypes.data, cols.ctypes.data,
                         rp.ctypes.data, bb.ctypes.data, x.ctypes.data, float(tolerance), int(max_iteration), int(stop),
                         ctypes.byref(it), ctypes.byref(res))
    _check(s, "fs_pcg_csr", (FS_NOT_CONVERGED,))
    return x, it.value, res.value, s


from .reference_api import CUDA_PCG_METHOD, EULERIAN_FLUID_SOLVER_3D, LINEAR_SOLVER, PROJECTION_3D  # noqa: E402,F401
