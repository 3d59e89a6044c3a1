// Headless driver around the reference solver, built only to produce golden
// vectors (test infrastructure, never part of the product path).
//
// It builds a SIMULATION_WORLD from a generated air/water .sim script exactly
// as the reference application does (SIMULATION_WORLD.h:InitializeFormScript),
// then lets the caller inject seeded interior fields and call single reference
// operators on them.  The golden vectors are made with number_of_threads = 1
// (thread_id 0: the reference's barriers are no-ops and its ordered partial
// sums plain sequential sums).  With number_of_threads = T in the script the
// timed operators run on T threads, each calling the reference routine with
// its thread_id, as MULTITHREADING::RunThreads does (used to time the
// reference's CPU path with every host thread).
//
// Field ids: 0 phi (cells), 1 u (x faces), 2 v (y faces), 3 w (z faces),
// 4 pressure (cells).  Arrays are interior values only, x fastest:
// idx = i + nx*(j + ny*k) with nx the extent of that field (n+1 on its own
// face axis).
#include <thread>
#include <vector>

#include "MARCHING_CUBES_ALGORITHM.h"
#include "SIMULATION_WORLD.h"

namespace {

struct RefCase {
  SIMULATION_WORLD world;
};

FIELD_STRUCTURE_3D<T>& field_of(RefCase* c, int id) {
  EULERIAN_FLUID_SOLVER_3D& s = c->world.eulerian_solver;
  switch (id) {
    case 0: return s.water_levelset->signed_distance_field;
    case 1: return *s.water_velocity_field_mac_x;
    case 2: return *s.water_velocity_field_mac_y;
    case 3: return *s.water_velocity_field_mac_z;
    default: return s.water_projection->pressure_field;
  }
}

template <class F>
void for_interior(FIELD_STRUCTURE_3D<T>& f, F&& body) {
  const GRID_STRUCTURE_3D& g = f.grid;
  long idx = 0;
  for (int k = g.k_start; k <= g.k_end; ++k)
    for (int j = g.j_start; j <= g.j_end; ++j)
      for (int i = g.i_start; i <= g.i_end; ++i) body(f.array_for_this(i, j, k), idx++);
}

// The reference's level set carries two ghost layers that its extrapolating
// ghost fill reads for layers >= 2 (FIELD_STRUCTURE_3D.h:1776-1830).  Filling
// them in place first, with the same routine, makes those reads well defined:
// the loop runs outward, so layer m reads the freshly written layer m-1.
void extrapolate_levelset_in_place(EULERIAN_FLUID_SOLVER_3D& s, int t = 0) {
  s.water_levelset->signed_distance_field.FillGhostCellsContinuousDerivativesFrom(t, s.water_levelset->arr, false);
}

void zero_ghost_velocities(EULERIAN_FLUID_SOLVER_3D& s, int t = 0) {
  s.vector_field_mac_ghost_x.FillGhostCellsZero(t, s.water_velocity_field_mac_x->array_for_this, true);
  s.vector_field_mac_ghost_y.FillGhostCellsZero(t, s.water_velocity_field_mac_y->array_for_this, true);
  s.vector_field_mac_ghost_z.FillGhostCellsZero(t, s.water_velocity_field_mac_z->array_for_this, true);
}

// body(thread_id) on every thread of the world's MULTITHREADING, as its
// RunThreads does; one thread runs inline.
template <class F>
void run_threads(RefCase* c, F&& body) {
  const int T = c->world.multithreading->num_threads;
  if (T <= 1) {
    body(0);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < T; ++t) th.emplace_back([&body, t] { body(t); });
  for (auto& x : th) x.join();
}

}  // namespace

extern "C" {

void* fsref_create(const char* sim_path) {
  RefCase* c = new RefCase;
  c->world.InitializeFormScript(sim_path);
  // ADVECTION_3D's constructor leaves its two boundary-mode flags
  // uninitialised (ADVECTION_3D.h:72-73, 87-97), and the first level-set
  // advection of a pipe run reads velocity_advection before any velocity
  // advection has set it; both start false here, the value they hold after
  // the first velocity advection of a run.  The flags matter in pipe mode only.
  if (ADVECTION_3D* adv = c->world.eulerian_solver.advecting_field_variables) {
    adv->levelset_advection = false;
    adv->velocity_advection = false;
  }
  return c;
}

void fsref_destroy(void* h) { delete static_cast<RefCase*>(h); }

void fsref_dims(void* h, int* out) {
  const GRID_STRUCTURE_3D& g = static_cast<RefCase*>(h)->world.eulerian_solver.base_grid;
  out[0] = g.i_res; out[1] = g.j_res; out[2] = g.k_res;
}

double fsref_dx(void* h) { return static_cast<RefCase*>(h)->world.eulerian_solver.base_grid.dx; }

void fsref_set(void* h, int id, const double* src) {
  for_interior(field_of(static_cast<RefCase*>(h), id), [&](T& v, long n) { v = src[n]; });
}

void fsref_get(void* h, int id, double* dst) {
  for_interior(field_of(static_cast<RefCase*>(h), id), [&](T& v, long n) { dst[n] = v; });
}

// Extrapolated level-set ghosts (three layers on the faces of the box), as
// the WENO5 stencil reads them.  Output layout: (n+6)^3, x fastest.
void fsref_levelset_ghost(void* h, double* dst) {
  EULERIAN_FLUID_SOLVER_3D& s = static_cast<RefCase*>(h)->world.eulerian_solver;
  extrapolate_levelset_in_place(s);
  s.scalar_field_ghost.FillGhostCellsContinuousDerivativesFrom(0, s.water_levelset->arr, true);
  const GRID_STRUCTURE_3D& g = s.base_grid;
  long idx = 0;
  for (int k = g.k_start - 3; k <= g.k_end + 3; ++k)
    for (int j = g.j_start - 3; j <= g.j_end + 3; ++j)
      for (int i = g.i_start - 3; i <= g.i_end + 3; ++i) dst[idx++] = s.scalar_field_ghost.array_for_this(i, j, k);
}

// One forward-Euler WENO5 level-set update (ADVECTION_METHOD_3D.h:42-279)
// with the ghost copy filled from the current level set by linear
// extrapolation and the MAC velocity ghosts zero-filled.
void fsref_weno5_levelset(void* h, double dt) {
  RefCase* c = static_cast<RefCase*>(h);
  EULERIAN_FLUID_SOLVER_3D& s = c->world.eulerian_solver;
  run_threads(c, [&](int t) {
    extrapolate_levelset_in_place(s, t);
    s.scalar_field_ghost.FillGhostCellsContinuousDerivativesFrom(t, s.water_levelset->arr, true);
    zero_ghost_velocities(s, t);
    ADVECTION_METHOD_3D<T>::WENO5th(t, s.water_levelset->signed_distance_field, s.scalar_field_ghost,
                                    s.vector_field_mac_ghost_x, s.vector_field_mac_ghost_y,
                                    s.vector_field_mac_ghost_z, dt, *c->world.multithreading,
                                    s.advecting_field_variables->epsilon);
  });
}

// One forward-Euler WENO5 update of the three MAC components.  own_ghost = 0
// reproduces ADVECTION_3D.h:317-319 (the x-component ghost copy is the
// stencil source for all three components); own_ghost = 1 gives each
// component its own ghost copy.
void fsref_weno5_velocity(void* h, double dt, int own_ghost) {
  RefCase* c = static_cast<RefCase*>(h);
  EULERIAN_FLUID_SOLVER_3D& s = c->world.eulerian_solver;
  MULTITHREADING& mt = *c->world.multithreading;
  const T eps = s.advecting_field_variables->epsilon_v;
  FIELD_STRUCTURE_3D<T>& gx = s.vector_field_mac_ghost_x;
  FIELD_STRUCTURE_3D<T>& gy = own_ghost ? s.vector_field_mac_ghost_y : s.vector_field_mac_ghost_x;
  FIELD_STRUCTURE_3D<T>& gz = own_ghost ? s.vector_field_mac_ghost_z : s.vector_field_mac_ghost_x;
  run_threads(c, [&](int t) {
    zero_ghost_velocities(s, t);
    ADVECTION_METHOD_3D<T>::WENO5th(t, *s.water_velocity_field_mac_x, gx, s.vector_field_mac_ghost_x, s.vector_field_mac_ghost_y, s.vector_field_mac_ghost_z, dt, mt, eps);
    ADVECTION_METHOD_3D<T>::WENO5th(t, *s.water_velocity_field_mac_y, gy, s.vector_field_mac_ghost_x, s.vector_field_mac_ghost_y, s.vector_field_mac_ghost_z, dt, mt, eps);
    ADVECTION_METHOD_3D<T>::WENO5th(t, *s.water_velocity_field_mac_z, gz, s.vector_field_mac_ghost_x, s.vector_field_mac_ghost_y, s.vector_field_mac_ghost_z, dt, mt, eps);
  });
}

// One forward-Euler ENO3 update of the three MAC components, each with its
// own zero-filled ghost copy (ADVECTION_3D.h:323-325).
void fsref_eno3_velocity(void* h, double dt) {
  RefCase* c = static_cast<RefCase*>(h);
  EULERIAN_FLUID_SOLVER_3D& s = c->world.eulerian_solver;
  MULTITHREADING& mt = *c->world.multithreading;
  run_threads(c, [&](int t) {
    zero_ghost_velocities(s, t);
    ADVECTION_METHOD_3D<T>::ENO3rd(t, *s.water_velocity_field_mac_x, s.vector_field_mac_ghost_x, s.vector_field_mac_ghost_x, s.vector_field_mac_ghost_y, s.vector_field_mac_ghost_z, dt, mt);
    ADVECTION_METHOD_3D<T>::ENO3rd(t, *s.water_velocity_field_mac_y, s.vector_field_mac_ghost_y, s.vector_field_mac_ghost_x, s.vector_field_mac_ghost_y, s.vector_field_mac_ghost_z, dt, mt);
    ADVECTION_METHOD_3D<T>::ENO3rd(t, *s.water_velocity_field_mac_z, s.vector_field_mac_ghost_z, s.vector_field_mac_ghost_x, s.vector_field_mac_ghost_y, s.vector_field_mac_ghost_z, dt, mt);
  });
}

// One reinitialisation block: S = phi0/sqrt(phi0^2 + dx^2) and
// iteration_number_for_reinitialization Sussman pseudo-steps of
// dtau = dx/scaling_number (EULERIAN_FLUID_SOLVER_3D.h Reinitialization).
// refresh_ghosts = 0 is the reference call as it stands (the level set's own
// ghost layers keep their value from before the block); refresh_ghosts = 1
// re-extrapolates them before every pseudo-step.
void fsref_reinitialization(void* h, double dt, int refresh_ghosts) {
  RefCase* c = static_cast<RefCase*>(h);
  EULERIAN_FLUID_SOLVER_3D& s = c->world.eulerian_solver;
  if (!refresh_ghosts) {
    run_threads(c, [&](int t) {
      extrapolate_levelset_in_place(s, t);
      s.Reinitialization(t, dt);
    });
    return;
  }
  extrapolate_levelset_in_place(s);
  const T fictious_dt = s.base_grid.dx / s.scaling_number_for_reinitialization;
  const GRID_STRUCTURE_3D& g = s.base_grid;
  for (int k = g.k_start; k <= g.k_end; ++k)
    for (int j = g.j_start; j <= g.j_end; ++j)
      for (int i = g.i_start; i <= g.i_end; ++i) {
        const T p = s.water_levelset->signed_distance_field(i, j, k);
        s.sign_function(i, j, k) = p / sqrt(POW2(p) + POW2(s.water_levelset->grid.dx));
      }
  for (int it = 0; it < s.iteration_number_for_reinitialization; ++it) {
    extrapolate_levelset_in_place(s);
    s.advecting_field_variables->ReinitializationBySussman(0, fictious_dt, s.sign_function);
  }
}

// PROJECTION_3D::Solve (PROJECTION_3D.h:416) on the injected phi and
// velocities; returns the PCG/CG iteration count of the pressure solve.
int fsref_projection(void* h, double dt) {
  RefCase* c = static_cast<RefCase*>(h);
  EULERIAN_FLUID_SOLVER_3D& s = c->world.eulerian_solver;
  run_threads(c, [&](int t) {
    extrapolate_levelset_in_place(s, t);
    s.water_projection->Solve(t, dt);
  });
  return s.water_projection->poisson_solver.linear_solver->num_iteration;
}

int fsref_poisson_rows(void* h) { return static_cast<RefCase*>(h)->world.eulerian_solver.water_projection->poisson_solver.A.N; }
int fsref_poisson_nnz(void* h) { return static_cast<RefCase*>(h)->world.eulerian_solver.water_projection->poisson_solver.A.nz; }

// CSR matrix, right-hand side (after mean removal) and solution of the last
// pressure solve, in the reference's own row numbering.
void fsref_poisson_csr(void* h, double* vals, int* cols, int* rowptr, double* b, double* x) {
  POISSON_SOLVER_3D& ps = static_cast<RefCase*>(h)->world.eulerian_solver.water_projection->poisson_solver;
  for (int n = 0; n < ps.A.nz; ++n) { vals[n] = ps.A.values[n]; cols[n] = ps.A.column_index[n]; }
  for (int r = 0; r <= ps.A.N; ++r) rowptr[r] = ps.A.row_ptr[r];
  for (int r = 0; r < ps.A.N; ++r) { b[r] = ps.b[r]; x[r] = ps.x[r]; }
}

// Divergence field of the last projection (cells, already divided by dt).
void fsref_divergence(void* h, double* dst) {
  PROJECTION_3D& p = *static_cast<RefCase*>(h)->world.eulerian_solver.water_projection;
  for_interior(p.divergence_field, [&](T& v, long n) { dst[n] = v; });
}

// Explicit variable-viscosity update (VISCOSITY_3D.h:452-563), in place.
void fsref_viscosity(void* h, double dt) {
  RefCase* c = static_cast<RefCase*>(h);
  EULERIAN_FLUID_SOLVER_3D& s = c->world.eulerian_solver;
  run_threads(c, [&](int t) {
    extrapolate_levelset_in_place(s, t);
    s.viscosity_solver->ApplyViscosity(t, s.epsilon_for_mollification, dt);
  });
}

// The same explicit update on fully defined inputs: the level set's first
// ghost layer (edges and corners included) is set from phi_g, the caller's
// one-layer ghosted copy ((n+2)^3 values, x fastest), and the first ghost
// layer of each velocity component is zeroed, so that every value the
// stencils read is given.  One thread.
void fsref_viscosity_ghosted(void* h, const double* phi_g, double dt) {
  RefCase* c = static_cast<RefCase*>(h);
  EULERIAN_FLUID_SOLVER_3D& s = c->world.eulerian_solver;
  FIELD_STRUCTURE_3D<T>& ls = s.water_levelset->signed_distance_field;
  const GRID_STRUCTURE_3D& g = ls.grid;
  long idx = 0;
  for (int k = g.k_start - 1; k <= g.k_end + 1; ++k)
    for (int j = g.j_start - 1; j <= g.j_end + 1; ++j)
      for (int i = g.i_start - 1; i <= g.i_end + 1; ++i) ls.array_for_this(i, j, k) = phi_g[idx++];
  FIELD_STRUCTURE_3D<T>* vel[3] = {s.water_velocity_field_mac_x, s.water_velocity_field_mac_y,
                                   s.water_velocity_field_mac_z};
  for (FIELD_STRUCTURE_3D<T>* f : vel) {
    const GRID_STRUCTURE_3D& fg = f->grid;
    for (int k = fg.k_start - 1; k <= fg.k_end + 1; ++k)
      for (int j = fg.j_start - 1; j <= fg.j_end + 1; ++j)
        for (int i = fg.i_start - 1; i <= fg.i_end + 1; ++i) {
          const bool inside = i >= fg.i_start && i <= fg.i_end && j >= fg.j_start && j <= fg.j_end &&
                              k >= fg.k_start && k <= fg.k_end;
          if (!inside) f->array_for_this(i, j, k) = 0.0;
        }
  }
  s.viscosity_solver->ApplyViscosity(0, s.epsilon_for_mollification, dt);
}

// Semi-implicit viscosity system for one MAC component through the reference
// builder and linear solver (POISSON_SOLVER_3D.h:3359-3496 + selected solver):
// (1 + sum c/dx^2) u_c - sum c_nb/dx^2 u_nb = explicit.  comp selects the
// face field; coef holds 6 interior arrays back to back; every interior face
// is an unknown, faces outside the component's grid are Dirichlet with the
// ghost value of the velocity field (zero here).  Returns the iteration count.
int fsref_semi_implicit_solve(void* h, int comp, const double* coef, const double* explicit_term, double* out) {
  EULERIAN_FLUID_SOLVER_3D& s = static_cast<RefCase*>(h)->world.eulerian_solver;
  FIELD_STRUCTURE_3D<T>& vel = field_of(static_cast<RefCase*>(h), comp);
  MULTITHREADING* mt = s.multithreading;
  FIELD_STRUCTURE_3D<T> cf[6], ex;
  FIELD_STRUCTURE_3D<int> bc;
  const GRID_STRUCTURE_3D& g = vel.grid;
  for (int m = 0; m < 6; ++m) {
    cf[m].Initialize(mt, g.i_res, g.j_res, g.k_res, g.i_start, g.j_start, g.k_start, g.x_min, g.y_min, g.z_min, g.x_max, g.y_max, g.z_max, 1);
    const long off = (long)m * g.ijk_res;
    for_interior(cf[m], [&](T& v, long n) { v = coef[off + n]; });
  }
  ex.Initialize(mt, g.i_res, g.j_res, g.k_res, g.i_start, g.j_start, g.k_start, g.x_min, g.y_min, g.z_min, g.x_max, g.y_max, g.z_max, 1);
  for_interior(ex, [&](T& v, long n) { v = explicit_term[n]; });
  bc.Initialize(mt, g.i_res, g.j_res, g.k_res, g.i_start, g.j_start, g.k_start, g.x_min, g.y_min, g.z_min, g.x_max, g.y_max, g.z_max, 1);
  for (int k = g.k_start - 1; k <= g.k_end + 1; ++k)
    for (int j = g.j_start - 1; j <= g.j_end + 1; ++j)
      for (int i = g.i_start - 1; i <= g.i_end + 1; ++i) {
        const bool inside = i >= g.i_start && i <= g.i_end && j >= g.j_start && j <= g.j_end && k >= g.k_start && k <= g.k_end;
        bc.array_for_this(i, j, k) = inside ? BC_FULL : BC_DIR;
      }
  POISSON_SOLVER_3D& ps = s.water_projection->poisson_solver;
  ps.SolveForViscosity(0, vel, cf[0], cf[1], cf[2], cf[3], cf[4], cf[5], bc, ex);
  for_interior(vel, [&](T& v, long n) { out[n] = v; });
  return ps.linear_solver->num_iteration;
}

// dt limit before the CFL factor (EULERIAN_FLUID_SOLVER_3D.h:2673-2785).
double fsref_cfl(void* h) { return static_cast<RefCase*>(h)->world.eulerian_solver.CFLOneTimeStep(); }

// Mean curvature of the level set (LEVELSET_3D.h ComputeCurvatures).
void fsref_curvature(void* h, double* dst) {
  EULERIAN_FLUID_SOLVER_3D& s = static_cast<RefCase*>(h)->world.eulerian_solver;
  extrapolate_levelset_in_place(s);
  s.water_levelset->ComputeCurvatures(0);
  for_interior(s.water_levelset->curvature, [&](T& v, long n) { dst[n] = v; });
}

// Plain linear solve through the reference's selected LINEAR_SOLVER on a
// caller-supplied CSR matrix (LINEAR_SOLVER.h:36).  Returns iterations.
int fsref_linear_solve(void* h, int n, int nnz, const double* vals, const int* cols, const int* rowptr,
                       const double* b, double* x) {
  EULERIAN_FLUID_SOLVER_3D& s = static_cast<RefCase*>(h)->world.eulerian_solver;
  MULTITHREADING* mt = s.multithreading;
  POISSON_SOLVER_3D& ps = s.water_projection->poisson_solver;
  CSR_MATRIX<T> A;
  A.Initialize(mt, n, nnz);
  mt->SplitDomainIndex1D(0, n);
  A.start_ix[0] = 0; A.end_ix[0] = n - 1; A.prev_row_array[0] = -1; A.values_ix_array[0] = 0;
  for (int r = 0; r < n; ++r)
    for (int q = rowptr[r]; q < rowptr[r + 1]; ++q) A.AssignValue(0, r, cols[q], vals[q]);
  VECTOR_ND<T> xv, bv;
  xv.Initialize(n, true);
  bv.Initialize(n);
  for (int r = 0; r < n; ++r) { xv[r] = x[r]; bv[r] = b[r]; }
  FIELD_STRUCTURE_3D<int>& bc = s.water_projection->boundary_condition_field;
  ps.linear_solver->Solve(0, A, xv, bv, bc);
  for (int r = 0; r < n; ++r) x[r] = xv[r];
  return ps.linear_solver->num_iteration;
}

// The level set in the reference's binary format (LEVELSET_3D::Write,
// LEVELSET_3D.h:1132-1160).
// LEVELSET_3D::ReinitializeByFastSweeping without its closing Update
// (normals and curvature, which can exit() on flat regions): a ghost fill,
// then FastSweepingMethod with sweep_direction = direction
// (LEVELSET_3D.h:601-610, 734-821).
void fsref_fast_sweeping(void* h, int direction) {
  RefCase* c = static_cast<RefCase*>(h);
  LEVELSET_3D& ls = *c->world.eulerian_solver.water_levelset;
  ls.sweep_direction = direction;
  run_threads(c, [&](int t) {
    ls.FillGhostCellsFrom(t, ls.phi, false);
    ls.FastSweepingMethod(t);
  });
}

// The level set's surface as WRITE_LEVELSET::WriteOBJ makes it
// (WRITE_LEVELSET.h:22-84): LEVELSET_3D::ComputeNormals (its UnitNormal
// orients the triangles), then MARCHING_CUBES_ALGORITHM::Polygonize.  Fills
// at most cap_v vertices (position xyz, normal nrm) and cap_t triangles
// (the OBJ's 1-based vertex indices); returns the vertex count and sets
// *ntri to the triangle count.
int fsref_marching_cubes(void* h, double* xyz, double* nrm, int cap_v, int* tri, int cap_t, int* ntri) {
  RefCase* c = static_cast<RefCase*>(h);
  LEVELSET_3D& ls = *c->world.eulerian_solver.water_levelset;
  run_threads(c, [&](int t) { ls.ComputeNormals(t); });
  MARCHING_CUBES_ALGORITHM mc;
  mc.Initialize(ls.multithreading, ls.grid);
  mc.Polygonize(static_cast<LEVELSET_OBJECT&>(ls));
  int nv = 0, nt = 0;
  for (int s = 0; s < mc.surfaces.num_elements; ++s) {
    TRIANGULAR_SURFACE* surf = mc.surfaces.values[s];
    for (VERTEX* v : surf->vertices) {
      if (nv < cap_v)
        for (int a = 0; a < 3; ++a) {
          xyz[3 * nv + a] = v->x[a];
          nrm[3 * nv + a] = v->n[a];
        }
      ++nv;
    }
  }
  for (int s = 0; s < mc.surfaces.num_elements; ++s) {
    TRIANGULAR_SURFACE* surf = mc.surfaces.values[s];
    for (TRIANGLE* t : surf->triangles) {
      if (nt < cap_t)
        for (int a = 0; a < 3; ++a) tri[3 * nt + a] = t->vertices[a]->index;
      ++nt;
    }
  }
  *ntri = nt;
  return nv;
}

// One frame of the reference application as its SIMULATION_MANAGER runs it
// (SIMULATION_WORLD::AdvanceOneFrame, SIMULATION_WORLD.h:320-331): the
// curvature, dt from the CFL condition on the head thread, then one whole
// timestep (EULERIAN_FLUID_SOLVER_3D::AdvanceOneTimeStepThread) on every
// thread of the world's MULTITHREADING, its pressure solves run to the
// script's tolerance.  The level set's ghost layers are extrapolated in place
// first so that the ghost fills read defined values.  Returns the PCG
// iteration count of the frame's last pressure solve; *dt_out gets the dt
// the frame used.  Used to time the reference's CPU step as a whole, with
// number_of_threads = 1: with 2 or 4 threads a whole frame of this build
// made no progress within a minute at 32^3 (the cause was not found; the
// reference's barrier, MULTITHREADING.h:105-118, waits on its condition
// without a predicate loop), while single operators run threaded.
int fsref_advance_frame(void* h, double* dt_out) {
  RefCase* c = static_cast<RefCase*>(h);
  EULERIAN_FLUID_SOLVER_3D& s = c->world.eulerian_solver;
  extrapolate_levelset_in_place(s);
  c->world.AdvanceOneFrame();
  if (dt_out) *dt_out = c->world.dt;
  return s.water_projection->poisson_solver.linear_solver->num_iteration;
}

// The pressure solver's stopping tolerance (LINEAR_SOLVER::SetTolerance):
// the reference stops its PCG when r.z < tolerance^2 (PCG_METHOD.cpp:87).
void fsref_set_pressure_tolerance(void* h, double tol) {
  static_cast<RefCase*>(h)->world.eulerian_solver.water_projection->poisson_solver.linear_solver->SetTolerance(tol);
}

void fsref_write_levelset(void* h, const char* path) {
  EULERIAN_FLUID_SOLVER_3D& s = static_cast<RefCase*>(h)->world.eulerian_solver;
  s.water_levelset->Write(path);
}

// ---- oil/water pipe mode (oil_water_simulation = true)

// The constants the reference derives from its pipe script
// (EULERIAN_FLUID_SOLVER_3D.h:496-514) and the cell grid:
// out = a, R1, m, eta, K, g, f, A, V0, J, Re, We, water_density, oil_density,
// water_viscosity, oil_viscosity, surface_tension, is_vertical, is_parallel,
// x_min, y_min, z_min, dx, dy, dz.
void fsref_pipe_params(void* h, double* out) {
  EULERIAN_FLUID_SOLVER_3D& s = static_cast<RefCase*>(h)->world.eulerian_solver;
  const GRID_STRUCTURE_3D& g = s.base_grid;
  const double v[] = {s.a, s.R1, s.m, s.eta, s.K, s.g, s.f, s.A, s.V0, s.J, s.Re, s.We, s.water_density,
                      s.oil_density, s.water_viscosity, s.oil_viscosity, s.surface_tension,
                      (double)s.is_vertical, (double)s.is_parallel, g.x_min, g.y_min, g.z_min, g.dx, g.dy, g.dz};
  for (size_t q = 0; q < sizeof(v) / sizeof(v[0]); ++q) out[q] = v[q];
}

// The cell-centred boundary level set (interior cells).
void fsref_boundary_levelset(void* h, double* dst) {
  EULERIAN_FLUID_SOLVER_3D& s = static_cast<RefCase*>(h)->world.eulerian_solver;
  for_interior(s.boundary_levelset->signed_distance_field, [&](T& v, long n) { dst[n] = v; });
}

// A ghosted copy used by the operators, with its three ghost layers:
// 0 the level-set ghost copy, 1-3 the MAC velocity ghost copies.
// Layout (extent + 6) per axis, x fastest.
void fsref_ghost_copy(void* h, int id, double* dst) {
  EULERIAN_FLUID_SOLVER_3D& s = static_cast<RefCase*>(h)->world.eulerian_solver;
  FIELD_STRUCTURE_3D<T>* f[] = {&s.scalar_field_ghost, &s.vector_field_mac_ghost_x, &s.vector_field_mac_ghost_y,
                                &s.vector_field_mac_ghost_z};
  FIELD_STRUCTURE_3D<T>& a = *f[id];
  const GRID_STRUCTURE_3D& g = a.grid;
  long idx = 0;
  for (int k = g.k_start - 3; k <= g.k_end + 3; ++k)
    for (int j = g.j_start - 3; j <= g.j_end + 3; ++j)
      for (int i = g.i_start - 3; i <= g.i_end + 3; ++i) dst[idx++] = a.array_for_this(i, j, k);
}

// The pipe's boundary level set on the faces of one component, as the
// advection's velocity set-up last computed it (ADVECTION_3D.h:380-430).
void fsref_boundary_faces(void* h, int comp, double* dst) {
  ADVECTION_3D& adv = *static_cast<RefCase*>(h)->world.eulerian_solver.advecting_field_variables;
  FIELD_STRUCTURE_3D<T>* f[] = {&adv.boundary_phi_x, &adv.boundary_phi_y, &adv.boundary_phi_z};
  for_interior(*f[comp], [&](T& v, long n) { dst[n] = v; });
}

// One of the advection's per-axis velocity ghost copies (ADVECTION_3D.h:
// 40-48; id = 3 * component + axis), with its three ghost layers, x fastest.
void fsref_adv_ghost(void* h, int id, double* dst) {
  ADVECTION_3D& adv = *static_cast<RefCase*>(h)->world.eulerian_solver.advecting_field_variables;
  FIELD_STRUCTURE_3D<T>* f[] = {&adv.velocity_field_mac_ghost_x_x, &adv.velocity_field_mac_ghost_x_y,
                                &adv.velocity_field_mac_ghost_x_z, &adv.velocity_field_mac_ghost_y_x,
                                &adv.velocity_field_mac_ghost_y_y, &adv.velocity_field_mac_ghost_y_z,
                                &adv.velocity_field_mac_ghost_z_x, &adv.velocity_field_mac_ghost_z_y,
                                &adv.velocity_field_mac_ghost_z_z};
  FIELD_STRUCTURE_3D<T>& a = *f[id];
  const GRID_STRUCTURE_3D& g = a.grid;
  long idx = 0;
  for (int k = g.k_start - 3; k <= g.k_end + 3; ++k)
    for (int j = g.j_start - 3; j <= g.j_end + 3; ++j)
      for (int i = g.i_start - 3; i <= g.i_end + 3; ++i) dst[idx++] = a.array_for_this(i, j, k);
}

// The fixed flags of a velocity component (1: the face keeps its value).
void fsref_fixed(void* h, int comp, unsigned char* dst) {
  EULERIAN_FLUID_SOLVER_3D& s = static_cast<RefCase*>(h)->world.eulerian_solver;
  FIELD_STRUCTURE_3D<T>* f[] = {s.water_velocity_field_mac_x, s.water_velocity_field_mac_y,
                                s.water_velocity_field_mac_z};
  FIELD_STRUCTURE_3D<T>& a = *f[comp];
  const GRID_STRUCTURE_3D& g = a.grid;
  long idx = 0;
  for (int k = g.k_start; k <= g.k_end; ++k)
    for (int j = g.j_start; j <= g.j_end; ++j)
      for (int i = g.i_start; i <= g.i_end; ++i) dst[idx++] = a.fixed(i, j, k) ? 1 : 0;
}

// ADVECTION_3D::Solve_Levelset in pipe mode (ADVECTION_3D.h:204-242): the
// velocity boundary set-up of the cylinder, the periodic ghost copy of the
// level set and the WENO5 update that skips cells outside the pipe.
void fsref_pipe_levelset_advection(void* h, double dt) {
  RefCase* c = static_cast<RefCase*>(h);
  EULERIAN_FLUID_SOLVER_3D& s = c->world.eulerian_solver;
  run_threads(c, [&](int t) { s.advecting_field_variables->Solve_Levelset(t, dt); });
}

// ADVECTION_3D::Solve_Velocity in pipe mode (ADVECTION_3D.h:244-358).
void fsref_pipe_velocity_advection(void* h, double dt) {
  RefCase* c = static_cast<RefCase*>(h);
  EULERIAN_FLUID_SOLVER_3D& s = c->world.eulerian_solver;
  run_threads(c, [&](int t) { s.advecting_field_variables->Solve_Velocity(t, dt); });
}

// EULERIAN_FLUID_SOLVER_3D::Reinitialization (EULERIAN_FLUID_SOLVER_3D.h:2198-2225).
void fsref_pipe_reinitialization(void* h, double dt) {
  RefCase* c = static_cast<RefCase*>(h);
  EULERIAN_FLUID_SOLVER_3D& s = c->world.eulerian_solver;
  run_threads(c, [&](int t) { s.Reinitialization(t, dt); });
}

// EULERIAN_FLUID_SOLVER_3D::ApplyGravity, the dimensionless forcing of the
// pipe (EULERIAN_FLUID_SOLVER_3D.h:2237-2432).
void fsref_pipe_gravity(void* h, double dt) {
  RefCase* c = static_cast<RefCase*>(h);
  EULERIAN_FLUID_SOLVER_3D& s = c->world.eulerian_solver;
  run_threads(c, [&](int t) { s.ApplyGravity(t, dt); });
}

// EULERIAN_FLUID_SOLVER_3D::Projection of the pipe (EULERIAN_FLUID_SOLVER_3D.h:
// 2226-2235 -> PROJECTION_3D::Solve, PROJECTION_3D.h:416-441): the cylinder's
// Neumann cells, the pipe divergence, the jump 1/We kappa, the PCG and the
// pipe velocity update.  Returns the PCG iteration count.
int fsref_pipe_projection(void* h, double dt) {
  RefCase* c = static_cast<RefCase*>(h);
  EULERIAN_FLUID_SOLVER_3D& s = c->world.eulerian_solver;
  run_threads(c, [&](int t) { s.Projection(t, dt); });
  return s.water_projection->poisson_solver.linear_solver->num_iteration;
}

// VISCOSITY_3D::ApplyViscosity of the pipe (the oil/water semi-implicit
// branch, VISCOSITY_3D.h:565-990) with the reference's epsilon 1.5 dx
// (EULERIAN_FLUID_SOLVER_3D.h:394), as Sourcing calls it (:2082).
void fsref_pipe_viscosity(void* h, double dt) {
  RefCase* c = static_cast<RefCase*>(h);
  EULERIAN_FLUID_SOLVER_3D& s = c->world.eulerian_solver;
  run_threads(c, [&](int t) { s.viscosity_solver->ApplyViscosity(t, s.epsilon_for_mollification, dt); });
}

// A coefficient field of the last semi-implicit viscosity solve: id = 7 *
// component + q, q = 0 the explicit term, 1..6 coef_1..coef_6 (interior
// faces of that component).
void fsref_visc_field(void* h, int id, double* dst) {
  VISCOSITY_3D& v = *static_cast<RefCase*>(h)->world.eulerian_solver.viscosity_solver;
  FIELD_STRUCTURE_3D<T>* f[] = {&v.explicit_term_x, &v.coef_1_x, &v.coef_2_x, &v.coef_3_x, &v.coef_4_x, &v.coef_5_x,
                                &v.coef_6_x, &v.explicit_term_y, &v.coef_1_y, &v.coef_2_y, &v.coef_3_y, &v.coef_4_y,
                                &v.coef_5_y, &v.coef_6_y, &v.explicit_term_z, &v.coef_1_z, &v.coef_2_z, &v.coef_3_z,
                                &v.coef_4_z, &v.coef_5_z, &v.coef_6_z};
  for_interior(*f[id], [&](T& x, long n) { dst[n] = x; });
}

// The jump condition and the divergence of the last projection (cells).
void fsref_projection_jc(void* h, double* dst) {
  PROJECTION_3D& p = *static_cast<RefCase*>(h)->world.eulerian_solver.water_projection;
  for_interior(p.jc_on_solution, [&](T& v, long n) { dst[n] = v; });
}

}  // extern "C"
