/*
 * fluid_b200.h - C ABI of the B200 (sm_100a) two-phase level-set solver
 * timestep: WENO5 level-set and velocity advection, Sussman
 * reinitialisation, semi-implicit viscosity and the variable-density
 * ghost-fluid pressure projection, all device resident.
 *
 * Every entry point returns an fs_status; none calls exit().  After any
 * status other than FS_CUDA_ERROR the context stays usable.  A context owns
 * one CUDA stream and all device memory of one simulation; it is not
 * re-entrant (one host thread at a time, as the reference's head-thread work
 * is).  Host arrays are borrowed only for the duration of a call.
 *
 * Array conventions (the reference's ARRAY_3D order, ARRAY_3D.h:98): x is the
 * fastest index.  Cell fields hold nx*ny*nz values; MAC face fields carry one
 * more entry along their own axis: u (nx+1)*ny*nz, v nx*(ny+1)*nz,
 * w nx*ny*(nz+1).  The grid is uniform with spacing dx on all axes; cell
 * (i,j,k) is centred at ((i+1/2)dx, (j+1/2)dx, (k+1/2)dx).  The phase with
 * phi <= 0 is the "negative" phase of fs_params.
 */
#ifndef FLUID_B200_H
#define FLUID_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fs_ctx fs_ctx;

typedef enum {
  FS_OK = 0,
  FS_INVALID_ARG = 1,     /* bad size, null pointer, unknown field or option */
  FS_OOM = 2,             /* device allocation failed; nothing was kept */
  FS_NOT_CONVERGED = 3,   /* an iterative solve stopped at its iteration cap */
  FS_NONFINITE = 4,       /* NaN/Inf detected in a residual or input */
  FS_CUDA_ERROR = 5,      /* a CUDA call failed; the context may be unusable */
  FS_TIMEOUT = 6,         /* a bounded device-side wait ran out */
  FS_NOT_SUPPORTED = 7
} fs_status;

typedef enum {
  FS_FIELD_PHI = 0,       /* level set, cells */
  FS_FIELD_U = 1,         /* x-velocity, x faces */
  FS_FIELD_V = 2,         /* y-velocity, y faces */
  FS_FIELD_W = 3,         /* z-velocity, z faces */
  FS_FIELD_PRESSURE = 4,  /* pressure of the last projection, cells */
  FS_FIELD_DIVERGENCE = 5, /* divergence/dt of the last projection's input, cells (download only) */
  FS_FIELD_ADJ_PHI = 6,   /* adjoint (bar) of phi, cells (FP64 in every context), see the adjoint entry points */
  FS_FIELD_ADJ_U = 7,     /* adjoint of u, x faces */
  FS_FIELD_ADJ_V = 8,     /* adjoint of v, y faces */
  FS_FIELD_ADJ_W = 9,     /* adjoint of w, z faces */
  FS_FIELD_CURVATURE = 10 /* mean curvature from the last fs_curvature or surface-tension projection (download only) */
} fs_field;

typedef enum {
  FS_PRECISION_FP64 = 0,        /* FP64 storage and arithmetic everywhere */
  FS_PRECISION_FP32_REFINE = 1  /* FP32 storage/stencils/inner PCG + FP64 defect correction */
} fs_precision;

typedef enum {
  FS_VELOCITY_WENO5 = 0,  /* VELOCITY_ADVECTION use_5th_weno_v (ADVECTION_METHOD_3D.h:42-279) */
  FS_VELOCITY_ENO3 = 1    /* use_3rd_eno_v, the reference scripts' choice (ADVECTION_METHOD_3D.h:1639-1934) */
} fs_velocity_scheme;

/* Preconditioner of the pressure solve. */
typedef enum {
  FS_PRECOND_DEFAULT = 0,     /* FP64: Jacobi (the reference's, PCG_METHOD.cpp:128-160); FP32_REFINE: red-black IC(0) */
  FS_PRECOND_JACOBI = 1,      /* z = r / diag in the solve precision */
  FS_PRECOND_JACOBI_BF16 = 2, /* FP32_REFINE: z = r * (1/diag rounded to bf16), 2 bytes per unknown */
  FS_PRECOND_RED_BLACK = 3,   /* FP32_REFINE: IC(0) in red-black order, i.e. the reference's commented-out
                                 incomplete Cholesky (PCG_METHOD.cpp:52-54, CSR_MATRIX.h:376) in multicolour
                                 ordering: the red cells are eliminated exactly and PCG runs on the black Schur
                                 complement S with the bf16 inverse of diag(S), the factor's black pivots */
  FS_PRECOND_RED_BLACK_JACOBI = 4 /* FP32_REFINE: the same reduced solve with the black cells' own bf16 1/diag */
} fs_preconditioner;

typedef enum {
  FS_STOP_RELATIVE = 0,   /* ||b - A p||_2 / ||b||_2 < tolerance */
  FS_STOP_ABSOLUTE = 1    /* r.z < tolerance^2, the reference's PCG test (PCG_METHOD.cpp:87) */
} fs_stop;

/* Behaviour switches; 0 is the corrected specification. */
enum {
  FS_FLAG_FAITHFUL_PROJECTION = 1 << 0, /* only w corrected + first-cell bottom face quirk (PROJECTION_3D.h:1188-1407) */
  FS_FLAG_REINIT_TYPO = 1 << 1,         /* reproduce the two sqrt(a^2)+b^2 leaves (ADVECTION_METHOD_3D.h:1463,1605) */
  FS_FLAG_LEVELSET_FORWARD_EULER = 1 << 2, /* order 3 advances phi by one Euler step (EULERIAN_FLUID_SOLVER_3D.h:1010) */
  FS_FLAG_CURVATURE_TYPO = 1 << 3, /* curvature as the reference computes it: factor 2 missing on py*pz*pyz and dz
                                      for 1/dz in the zero-gradient fallback (LEVELSET_3D.h:1033,1037) */
  FS_FLAG_SORT_TYPO = 1 << 4,      /* fast sweeping with the reference's INCREASING_SORT3, whose c < b < a branch
                                      leaves a2 stale (MACROS.h:61-68); sweeps then run sequentially */
  FS_FLAG_VISCOSITY_IN_PLACE = 1 << 5 /* explicit viscosity as the reference runs it: x, then y, then z, in place
                                         in (k, j, i) order, wall faces included, its shear-term velocity indices
                                         (VISCOSITY_3D.h:452-563) */
};

typedef struct {
  int nx, ny, nz;
  double dx;
} fs_grid_desc;

typedef struct {
  double rho_neg, rho_pos;          /* density of the phase at phi <= 0 / phi > 0 */
  double mu_neg, mu_pos;            /* dynamic viscosity, same convention */
  double gravity[3];                /* gravity (the reference's default is (0,-9.8,0)) */
  double weno_epsilon;              /* LEVELSET_ADVECTION.epsilon (also the reinit clamp) */
  int reinit_iterations;            /* iteration_number_for_reinitialization */
  int reinit_scaling;               /* scaling_number_for_reinitialization: dtau = dx/scaling */
  int order;                        /* order_for_time_advancing: 1, 2 or 3 */
  int precision;                    /* fs_precision */
  int stop;                         /* fs_stop for the pressure solve */
  double tolerance;                 /* pressure tolerance (relative divergence in FP32_REFINE) */
  int max_iteration;                /* PCG iteration cap per solve (inner cap in FP32_REFINE) */
  double inner_tolerance;           /* FP32_REFINE: residual reduction one FP32 Krylov sequence is trusted
                                       for before it restarts from the FP64 residual (default 1e-3) */
  int max_outer;                    /* FP32_REFINE: unused (kept for layout); the iteration cap applies */
  int viscosity;                    /* 0: off, 1: semi-implicit, 2: explicit (the reference's air/water update,
                                       VISCOSITY_3D.h:452-563; its dt limit enters fs_cfl_dt) */
  double viscosity_tolerance;       /* relative residual of each viscosity solve */
  int viscosity_max_iteration;
  double cfl;                       /* CFL number used by fs_cfl_dt */
  int flags;                        /* FS_FLAG_* */
  double surface_tension;           /* sigma: the pressure jump sigma*kappa across the interface (0: none) */
  int velocity_scheme;              /* fs_velocity_scheme of the velocity self-advection */
  double velocity_epsilon;          /* VELOCITY_ADVECTION.epsilon of the WENO5 weights (0: weno_epsilon) */
  int fast_sweeping;                /* fastsweeping_reinitialization: each reinitialisation block starts with
                                       fs_fast_sweeping(ctx, -1, 1) (EULERIAN_FLUID_SOLVER_3D.h:2202-2205) */
  int pressure_preconditioner;      /* fs_preconditioner of the pressure solve */
  double reliable_delta;            /* FP32_REFINE: the true FP64 residual replaces the recursive one each time the
                                       latter drops by this factor (0: 0.1) */
  int flux_arithmetic;              /* FP32_REFINE pressure SpMV: each face flux a (x_c - x_n) formed in 0: FP64,
                                       1: FP32 and summed in FP64, 2: FP32 throughout (default) */
  int verbose;                      /* 1: solver progress on stderr */
  int host_loop;                    /* 0 (default): each Krylov solve is one CUDA graph launch (a conditional while
                                       node repeating 16-iteration batches); 1: the same kernels launched from the
                                       host, 16 iterations between polls of the solver state (for profilers that do
                                       not descend into conditional graph nodes) */
  /* Oil/water pipe mode, the reference's oil_water_simulation with a vertical
     pipe (PIPE_OPTIONS.is_vertical): 0 (default) the air/water box with walls;
     1 a pipe along y, periodic in y with the reference's node convention (cell
     0 and cell ny-1 are one point), its wall at sqrt(x^2 + z^2) = pipe_radius.
     Built for the level-set advection, the reinitialisation, the ENO3 velocity
     advection, the body force and the projection (fs_advect_levelset,
     fs_reinitialize, fs_advect_velocity with velocity_scheme
     FS_VELOCITY_ENO3, fs_apply_gravity, fs_project: the cylinder's cells are
     the unknowns, the cells outside it Neumann cells, rho_neg and rho_pos
     the dimensionless densities 1 and water_density/oil_density, the
     pressure solve with the Jacobi preconditioners only), the CFL time
     step (fs_cfl_dt: the dimensionless form's terms, no viscous term) and
     the whole step with viscosity = 0 (fs_step: the reference's step with
     is_sourcing_active = false); the viscosity (fs_viscosity, fs_step with
     viscosity != 0) and the adjoints return FS_NOT_SUPPORTED in this mode.
     Fixed at creation. */
  int pipe;
  double pipe_radius;               /* a: the wall radius in units of the core radius R1 */
  double grid_min[3], grid_max[3];  /* the script's base_grid_min and base_grid_max: cell (i,j,k) sits at
                                       grid_min + (i,j,k) (grid_max - grid_min)/(n - 1), as in the reference */
  double pipe_R1;                   /* R1 = R2/a */
  double pipe_V0;                   /* V0, the velocity scale of the dimensionless form */
  double pipe_f;                    /* f, the driving pressure gradient */
  double pipe_eta;                  /* eta, the density ratio of the dimensionless form */
  double pipe_oil_density;          /* oil_density */
  double pipe_We;                   /* We, the Weber number of the dimensionless form: the pipe's projection
                                       carries the jump condition kappa/We (PROJECTION_3D.h:758-762) */
} fs_params;

typedef struct {
  int iterations;           /* PCG iterations (sum of inner iterations in FP32_REFINE) */
  int outer_iterations;     /* FP32_REFINE defect corrections (1 in FP64) */
  double rel_residual;      /* final ||b - A p||_2/||b||_2 in FP64 */
  double rz;                /* final r.z of the last PCG */
  double div_l2, div_linf;  /* divergence of the corrected velocity (cells, not scaled by dt) */
  float ms;                 /* device time of the call */
} fs_solve_report;

typedef struct {
  int pcg_iterations;       /* over all projections of the step */
  int outer_iterations;
  int viscosity_iterations;
  int projections;
  double max_rel_residual;  /* worst pressure residual of the step */
  double div_l2, div_linf;  /* divergence after the last projection */
  float ms;                 /* device time of the step */
  float pcg_ms;             /* device time inside the pressure PCG loops (FP32 inner loops in FP32_REFINE) */
  int pcg_launched_iterations; /* PCG iterations whose kernels ran in those loops (incl. the idle tail of the last batch) */
  int64_t kernel_launches;  /* kernels launched by the step (graph nodes counted individually) */
} fs_step_report;

/* Defaults that reproduce the reference's script defaults where it has them
 * (EULERIAN_FLUID_SOLVER_3D.h:192-260, PROJECTION_3D.h:178-230) and the
 * configuration's values elsewhere. */
void fs_params_default(fs_params* p);
const char* fs_status_str(fs_status s);
const char* fs_last_error(void);

/* Context life cycle (replaces EULERIAN_FLUID_SOLVER_3D::InitializeFromScriptBlock,
 * EULERIAN_FLUID_SOLVER_3D.h:192).  Allocates every device buffer up front. */
fs_status fs_create(const fs_grid_desc* grid, const fs_params* params, fs_ctx** out);
fs_status fs_destroy(fs_ctx* ctx);
fs_status fs_set_params(fs_ctx* ctx, const fs_params* params);
fs_status fs_memory_bytes(const fs_ctx* ctx, int64_t* bytes);

/* Host <-> device copies of one field (FP64 host values; converted to the
 * context's storage precision).  Non-NULL strides give element strides of
 * the host array in x, y, z (default: packed). */
fs_status fs_upload(fs_ctx* ctx, int field, const double* host, const int64_t* strides);
fs_status fs_download(fs_ctx* ctx, int field, double* host, const int64_t* strides);
/* Same, from/to device memory the caller owns (FP64, packed). */
fs_status fs_upload_device(fs_ctx* ctx, int field, const double* dev);
fs_status fs_download_device(fs_ctx* ctx, int field, double* dev);

/* One timestep (EULERIAN_FLUID_SOLVER_3D::AdvanceOneTimeStepThread,
 * EULERIAN_FLUID_SOLVER_3D.h:803-1111). */
fs_status fs_step(fs_ctx* ctx, double dt, fs_step_report* report);
/* CFL-limited dt times params.cfl (CFLOneTimeStep, EULERIAN_FLUID_SOLVER_3D.h:2673-2785). */
fs_status fs_cfl_dt(fs_ctx* ctx, double* dt);

/* Mean curvature of the current level set (LEVELSET_3D::ComputeCurvatures,
 * LEVELSET_3D.h:963) into FS_FIELD_CURVATURE; kappa_max (may be NULL) gets
 * max |kappa| over cells with |phi| < 0.1, the value the CFL condition uses. */
fs_status fs_curvature(fs_ctx* ctx, double* kappa_max);

/* Single operators of the step, on the context's current fields. */
/* PROJECTION_3D::Solve (PROJECTION_3D.h:416). */
fs_status fs_project(fs_ctx* ctx, double dt, fs_solve_report* report);
/* One forward-Euler WENO5 level-set update (ADVECTION_3D::Solve_Levelset, ADVECTION_3D.h:204). */
fs_status fs_advect_levelset(fs_ctx* ctx, double dt);
/* One forward-Euler WENO5 update of u, v, w (ADVECTION_3D::Solve_Velocity, ADVECTION_3D.h:244). */
fs_status fs_advect_velocity(fs_ctx* ctx, double dt);
/* One reinitialisation block (EULERIAN_FLUID_SOLVER_3D::Reinitialization, :2198). */
fs_status fs_reinitialize(fs_ctx* ctx);
/* EULERIAN_FLUID_SOLVER_3D::ApplyGravity (EULERIAN_FLUID_SOLVER_3D.h:2237-2432):
   u += dt g on interior faces in the box; in pipe mode the dimensionless body
   force on the y faces inside the pipe, R1/V0^2 (dt g_y + dt f/(oil_density
   rho_f)), rho_f = 1 + (eta - 1) H(phi_f), except the centre-line faces the
   reference holds fixed (i = (nx-1)/2, k = (nz-1)/2). */
fs_status fs_apply_gravity(fs_ctx* ctx, double dt);
/* LEVELSET_3D::ReinitializeByFastSweeping (LEVELSET_3D.h:601-610) on phi,
 * without the closing normals and curvature: the set-up (cells beyond
 * 20 dx and cells next to the interface fixed, the others reset to
 * +-20 dx), then `pairs` pairs of Gauss-Seidel sweeps, the first in sweep
 * direction `direction` (0..3; -1: the context's counter, which then
 * advances by one as the reference's sweep_direction does).  pairs = 1 is
 * the reference's call; pairs = 4 sweeps all eight octants after one
 * set-up.  FS_NONFINITE with FS_FLAG_SORT_TYPO when the reference's sort
 * reads its uninitialised a2 on this input. */
fs_status fs_fast_sweeping(fs_ctx* ctx, int direction, int pairs);

/* The zero level set of phi as a closed triangle mesh: the surface that
 * WRITE_LEVELSET::WriteOBJ writes (WRITE_LEVELSET.h:22-84), by marching
 * cubes over the cells with corners sampled as the reference samples them
 * (MARCHING_CUBES_ALGORITHM.h:146-166, 497-757).  Polygonises on the device
 * and keeps the mesh in the context; returns its vertex and triangle
 * counts. */
fs_status fs_surface(fs_ctx* ctx, int64_t* n_vertices, int64_t* n_triangles);
/* The mesh of the last fs_surface into host buffers sized from its counts:
 * xyz [3 nv] and normals [3 nv] (x, y, z per vertex; either may be NULL),
 * triangles [3 nt] with 1-based vertex numbers (may be NULL). */
fs_status fs_surface_download(fs_ctx* ctx, double* xyz, double* normals, int32_t* triangles);
/* fs_surface, then a Wavefront OBJ file: v and vn lines, faces "f a//a b//b c//c". */
fs_status fs_write_obj(fs_ctx* ctx, const char* path);
/* Semi-implicit viscosity of u, v, w (VISCOSITY_3D::ApplyViscosity, VISCOSITY_3D.h:448). */
fs_status fs_viscosity(fs_ctx* ctx, double dt, int* iterations);

/* LINEAR_SOLVER::Solve plugin (LINEAR_SOLVER.h:36): Jacobi-PCG on a CSR
 * matrix given on the host, x in/out (initial guess in).  Runs on the
 * context's stream with its own temporary device buffers. */
fs_status fs_pcg_csr(fs_ctx* ctx, int n, int nnz, const double* values, const int* column_index,
                     const int* row_ptr, const double* b, double* x, double tolerance, int max_iteration,
                     int stop, int* iterations, double* residual);

/* State I/O.  The level set in the reference's binary format
 * (LEVELSET_3D::Write / Read, LEVELSET_3D.h:1132-1200): int32 i_start,
 * j_start, k_start, i_res, j_res, k_res, float64 x_min, y_min, z_min, x_max,
 * y_max, z_max, int32 ghost_width, then phi as float64, x fastest.  grid_min
 * (may be NULL: the origin) is the position of cell (0,0,0); reading checks
 * the resolution and the spacing against the context and returns grid_min. */
fs_status fs_write_levelset(fs_ctx* ctx, const char* path, const double* grid_min);
fs_status fs_read_levelset(fs_ctx* ctx, const char* path, double* grid_min);
/* Checkpoint and resume of the step state (phi, u, v, w, pressure) in this
 * library's own format (magic "FSB200ST", version 1, grid, then the fields
 * as float64).  No counterpart in the reference, which has no restart. */
fs_status fs_write_state(fs_ctx* ctx, const char* path);
fs_status fs_read_state(fs_ctx* ctx, const char* path);

/* Adjoints (vector-Jacobian products) of the step and of its operators.
 * No counterpart in the reference, which has no derivatives; they are part
 * of this library's differentiable-simulation interface.
 *
 * The context's FS_FIELD_ADJ_* fields hold bars: on entry the bars of an
 * operator's outputs, on return the bars of its inputs.  A field that is both
 * input and output has its bar replaced; an input that is not an output has
 * its bar added to (so compositions accumulate).  The primal fields
 * (PHI, U, V, W) must hold the operator's INPUT state; the forward is
 * recomputed inside the call.  The density bars d/d(rho_neg), d/d(rho_pos)
 * accumulate in the context across calls (fs_adjoint_density_bars reads them,
 * fs_adjoint_reset clears them and the adjoint fields).
 *
 * Derivatives are those of the discrete operators as computed, with the
 * upwind sides of WENO5, the Godunov branches and sign clamp of the Sussman
 * step and the phase (sign of phi) of each cell frozen at their forward
 * values; the pressure and viscosity solves are differentiated as exact
 * solves (a second solve with the same symmetric operator).  dt is a
 * constant (not differentiated through the CFL condition).
 * FP64 and FP32_REFINE contexts: the forward states and the tape are kept in
 * the context's storage precision, every bar, derivative and sum is FP64,
 * and the transposed pressure solve uses the context's own solver (FP64
 * PCG, or the FP32 solve with FP64 defect correction).  The corrected
 * projection, WENO5 velocity advection, the semi-implicit or no viscosity,
 * no surface tension and Sussman reinitialisation only (FS_NOT_SUPPORTED
 * otherwise).  A transposed solve that stops before its tolerance leaves
 * inexact bars and the call returns FS_NOT_CONVERGED after completing.
 * The first call allocates the adjoint buffers; fs_step_adjoint also
 * allocates its tape (about 30 + 3*reinit_iterations fields). */
fs_status fs_adjoint_reset(fs_ctx* ctx);
fs_status fs_adjoint_density_bars(fs_ctx* ctx, double* rho_neg_bar, double* rho_pos_bar);
/* Whole step: ADJ_* = bars of the step's output -> bars of its input.  The
 * primal fields end in the step's OUTPUT state (the forward ran once). */
fs_status fs_step_adjoint(fs_ctx* ctx, double dt, fs_step_report* report);
/* Operator adjoints; the primal fields are left as they were. */
fs_status fs_advect_levelset_adjoint(fs_ctx* ctx, double dt);  /* phi -> phi (u, v, w bars added) */
fs_status fs_advect_velocity_adjoint(fs_ctx* ctx, double dt);  /* (u, v, w) -> (u, v, w) */
fs_status fs_reinitialize_adjoint(fs_ctx* ctx);                /* phi -> phi, one block */
fs_status fs_viscosity_adjoint(fs_ctx* ctx, double dt);        /* (u, v, w) -> (u, v, w); phi and density bars added */
fs_status fs_project_adjoint(fs_ctx* ctx, double dt);          /* (u, v, w) -> (u, v, w); phi and density bars added */

/* Allocation-free fs_pcg_csr, for callers that cannot allocate device
 * memory during a solve (a host whose device memory pool is owned by another
 * runtime, a real-time loop that must not take cudaMalloc's implicit
 * synchronisation).  No counterpart in the reference: it is an addition of
 * this library.  Every pointer is DEVICE memory the caller owns: the CSR
 * matrix (values [nnz], column_index [nnz], row_ptr [n + 1]), b, and x
 * (initial guess in, result out); stream may be NULL (the legacy default
 * stream).  The working vectors live in one fixed device array of the
 * library (n <= 262144 rows, about 8.4 MB on every GPU that loads the
 * library, kept until the process exits); larger systems are rejected with
 * FS_INVALID_ARG.  Each call looks up that array's device address with the
 * caller's device current (no allocation); the first call on a device also
 * loads the library's device code there, so make it before any stream
 * capture.  The call waits on `stream` between batches of 16 iterations and
 * returns when the solve has ended.  All calls share the array: calls that
 * overlap on the GPU (from several host threads or streams) race and must
 * not be issued.  The matrix is checked on the device before it is used: a
 * row_ptr entry outside [0, nnz], a decreasing row_ptr or a column index
 * outside [0, n) ends the call with FS_INVALID_ARG, reading nothing outside
 * the arrays and leaving x unchanged.  Every row needs a nonzero diagonal
 * (a zero diagonal ends the solve with FS_NONFINITE).  max_iteration = 0
 * runs no iteration (x unchanged, FS_NOT_CONVERGED unless b - A x already
 * meets the test).  After FS_CUDA_ERROR, kernels of the call may still be
 * queued on `stream`: synchronise it before reusing x or calling again.
 * No device or host memory is allocated. */
fs_status fs_pcg_csr_noalloc(int n, int nnz, const double* values, const int* column_index, const int* row_ptr,
                             const double* b, double* x, double tolerance, int max_iteration, int stop,
                             void* stream, int* iterations, double* residual);

#ifdef __cplusplus
}
#endif

#endif /* FLUID_B200_H */
