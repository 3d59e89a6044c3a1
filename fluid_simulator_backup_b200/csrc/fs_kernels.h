// Host-side declarations of the kernel launchers (one translation unit per
// kernel family; all are explicitly instantiated for float and double).
#pragma once

#include "fs_common.cuh"

namespace fsb {

// ---- stencil family (fs_stencil.cu)
template <class T> void fill_extrap(T* f, const Lay& L, cudaStream_t s);

// Geometry of the oil/water vertical pipe (fs_pipe.cu): the wall radius and,
// for the cell grid (0) and the x, y, z face grids (1..3), the x and z
// position of index 0 and the spacing, computed as the reference computes
// its grids (GRID_STRUCTURE_3D.h:91-137).
struct PipeGeom {
  int on;  // 0: the box
  double a;
  double ox[4], oz[4], hx[4], hz[4];
  // the first unknown of the pressure system in the reference's row order
  // (k, j, i): the cell that carries the faithful projection's deflation
  int fi, fj, fk;
  int64_t cells;  // unknowns of the pressure system (cells inside the pipe)
};
// sqrt(x^2 + z^2) - a at point (i, k) of grid g, in the reference's rounding
__device__ __forceinline__ double pipe_wall_distance(const PipeGeom& G, int g, int i, int k) {
  const double X = __dadd_rn(G.ox[g], __dmul_rn((double)i, G.hx[g]));
  const double Z = __dadd_rn(G.oz[g], __dmul_rn((double)k, G.hz[g]));
  return __dsub_rn(sqrt(__dadd_rn(__dmul_rn(X, X), __dmul_rn(Z, Z))), G.a);
}
// A cell of the box that is no unknown of the pipe's pressure system: wall
// distance > 0, the reference's Neumann cells (PROJECTION_3D.h:1017-1040).
// Always false in the box.
__device__ __forceinline__ bool pipe_solid(const PipeGeom& G, int i, int k) {
  return G.on && pipe_wall_distance(G, 0, i, k) > 0.0;
}
// periodic ghosts along y of a cell field (cell 0 and cell ny-1 are one
// point); the x and z ghost layers become 0
template <class T> void fill_periodic_y(T* f, const Lay& L, cudaStream_t s);
// the velocities the pipe's level-set advection reads (ghost copies g*) and
// the zeroing of u and w outside the pipe
template <class T>
void pipe_levelset_velocities(T* u, T* v, T* w, T* ug, T* vg, T* wg, const Lay& Lu, const Lay& Lv, const Lay& Lw,
                              const PipeGeom& G, cudaStream_t s);
// the ghost copies of the pipe's velocity advection: per component the masked
// periodic copy with its wall extrapolation (gen) and the copies guarded for
// the ENO3 stencils along x (gx) and z (gz); returns the kernels launched
template <class T>
int pipe_velocity_copies(const T* const comp[3], T* const gen[3], T* const gx[3], T* const gz[3], const Lay* const L[3],
                         const PipeGeom& G, cudaStream_t s);
// the pipe's ENO3 self-advection of one component, in place
template <class T>
void eno3_pipe(T* comp, const T* gen, const T* gx, const T* gz, const T* ug, const T* vg, const T* wg, const Lay& Lc,
               const Lay& Lu, const Lay& Lv, const Lay& Lw, int axis, const PipeGeom& G, double dx, double dt,
               cudaStream_t s);
// the pipe's dimensionless body force on v (phi with periodic y ghosts)
template <class T>
void pipe_forcing(T* v, const T* phi, const Lay& Lv, const Lay& Lc, const PipeGeom& G, double coef, double gdt,
                  double fdt, double oil_density, double eta, double eps, cudaStream_t s);
// the pipe's projection: b = -(div u)/dt on the unknowns from the pipe's
// velocity copies (0 elsewhere) with sum(b) in scalars[0]; the pipe's
// velocity update and its periodic rows (pressure p in FP64, kappa the
// curvature, jc = sigma kappa)
template <class T>
void pipe_divergence_rhs(const T* u, const T* v, const T* w, const Lay& Lc, const Lay& Lu, const Lay& Lv,
                         const Lay& Lw, const PipeGeom& G, double dx, double dt, double* b, double* div_out,
                         double* partials, unsigned int* ticket, double* scalars, cudaStream_t s);
template <class T>
void pipe_velocity_correct(T* u, T* v, T* w, const double* p, const T* phi, const double* kappa, const Lay& Lc,
                           const Lay& Lu, const Lay& Lv, const Lay& Lw, const PipeGeom& G, double dx, double dt,
                           double rho_neg, double rho_pos, double sigma, cudaStream_t s);
template <class T>
void weno5_levelset(const T* src, const T* base, T* out, const T* u, const T* v, const T* w, const Lay& L,
                    const Lay& Lu, const Lay& Lv, const Lay& Lw, double dx, double eps, double dt, double c0, double c1,
                    cudaStream_t s, const PipeGeom* pipe = nullptr);
template <class T>
void weno5_mac(const T* comp, T* out, const T* u, const T* v, const T* w, const Lay& Lc, const Lay& Lu, const Lay& Lv,
               const Lay& Lw, int axis, double dx, double eps, double dt, cudaStream_t s);
template <class T>
void eno3_mac(const T* comp, T* out, const T* u, const T* v, const T* w, const Lay& Lc, const Lay& Lu, const Lay& Lv,
              const Lay& Lw, int axis, double dx, double dt, cudaStream_t s);
template <class T> void sign_function(const T* phi, T* sgn, const Lay& L, double dx, cudaStream_t s);
// The zero level set as a triangle mesh in device memory (fs_surface.cu).
struct SurfaceMesh {
  double* xyz = nullptr;      // [nv][3]
  double* normals = nullptr;  // [nv][3]
  int* tri = nullptr;         // [nt][3], 1-based vertex numbers
  int64_t nv = 0, nt = 0;
  void release();
};
template <class T>
cudaError_t polygonize(const T* phi, const Lay& L, double dx, SurfaceMesh* mesh, cudaStream_t s);
// LEVELSET_3D::ReinitializeByFastSweeping from `in` into `out` (interior
// and face ghosts; `in` is not written): the set-up, then `pairs` sweep
// pairs starting at sweep direction `direction` (the reference runs one per
// call).  typo: the reference's sort with its stale a2, sequentially;
// *stale_read is set when that sort reads a2 before the sweep wrote it.
// Returns the number of kernels launched.
template <class T>
int fast_sweeping(const T* in, T* out, unsigned char* fixed, const Lay& L, double dx, int direction, int pairs,
                  int typo, int* stale_read, cudaStream_t s);
template <class T>
void sussman_step(const T* src, const T* sgn, const T* base, T* out, const Lay& L, double dx, double eps, double dtau,
                  double c0, double c1, int typo, cudaStream_t s);
template <class T> void axpby(T* out, const T* x, const T* y, double a, double b, const Lay& L, cudaStream_t s);
template <class T> void add_const_faces(T* f, const Lay& L, int axis, double value, int skip_walls, cudaStream_t s);
template <class T> void zero_walls(T* f, const Lay& L, int axis, cudaStream_t s);

// ---- Krylov solver state shared by the pressure and viscosity solves
struct PcgState {
  double rz, pq, rr, bb, beta, tol;
  double best_rr;         // smallest r.r seen
  double max_rr;          // r.r of the last true residual (reference of the reliable-update trigger)
  double rz_prev;         // r.z at the start of the last accepted step
  double reliable_delta;  // pause for a true residual when ||r|| < delta*max||r|| (0: never)
  double alpha;           // step length of the current iteration (set by the SpMV)
  int iter, max_iter, done, criterion, status, stall;
  int stall_limit;  // iterations without a 1% improvement of best_rr before giving up (0: never)
  int x_pending;    // alpha is set and x += alpha p is still due (applied by the direction update)
  unsigned int ticket;
  unsigned int ticket2;  // completion count of the direction update
};

// STAGNATED: the iteration can make no further progress in its arithmetic
// (p.Ap <= 0 or no improvement for stall_limit iterations); the iterate is
// kept and the caller decides.  RELIABLE_UPDATE: paused (done = 2) for the
// caller to replace the recursive residual by the true one.
enum { PCG_RUNNING = 0, PCG_CONVERGED = 1, PCG_MAXITER = 2, PCG_NONFINITE = 3, PCG_STAGNATED = 4,
       PCG_RELIABLE_UPDATE = 5 };

// Seven-point symmetric operator on a padded layout:
// (A x)_c = diag_c x_c - sum_d (a_d[c] x_{c-e_d} + a_d[c+e_d] x_{c+e_d});
// a_d[c] couples c-e_d and c.  Couplings across walls are zero, so ghost
// values of x never contribute.
// flux_form != 0 applies the operator as a sum of face fluxes,
// (A x)_c = sum_faces a_f (x_c - x_nb) + extra0 x_c (extra0 only at the first
// cell, the deflation term), which avoids the catastrophic cancellation of
// diag*x_c - sum a x_nb for smooth x: in FP32 the relative error of A x then
// grows like eps*n instead of eps*cond(A).  The diagonal is still used for
// the Jacobi preconditioner.  flux_form requires diag = sum of the face
// couplings everywhere except the first cell (true for the pressure matrix).
template <class V> struct Op7 {
  const V* ax;
  const V* ay;
  const V* az;
  const V* diag;
  Lay L;
  int flux_form = 0;
  const double* extra0 = nullptr;  // device scalar: diag - sum of couplings at the deflated cell
  int64_t c_extra = -1;            // the deflated cell (-1: cell (0,0,0) of the box)
  // flux form with FP32 vectors: 0 sums FP64 fluxes formed from exact FP64
  // differences and products; 1 forms each flux in FP32 (difference and
  // product correctly rounded) and sums them in FP64; 2 does all in FP32.
  // Each FP32 flux a (x_c - x_n) is exact to 2 eps32 of itself (the stored x
  // are exact inputs, so the difference is correctly rounded); the sum of six
  // loses eps32 * sum|flux| to cancellation, an inexact matrix-vector product
  // that the mixed solve's reliable updates (true residual in FP64) absorb:
  // at 256^3 mode 2 needs the same iterations as mode 0 and avoids the
  // FP32->FP64 conversions that bound the SpMV's issue rate.
  int flux32 = 0;
  // Jacobi preconditioner of the FP32 pressure solve: z = r * dinv16 with
  // 1/diag rounded to bf16 (2 bytes per unknown read twice per iteration
  // instead of 4).  Any fixed SPD diagonal is a valid preconditioner; a
  // 2^-9 relative perturbation of it moves the condition number of the
  // preconditioned system by under 0.5 %.
  const unsigned short* dinv16 = nullptr;  // bf16 bit patterns of 1/diag
};

template <class V, class R = V>
void pcg_init(const Op7<V>& A, const R* b, R* x, R* r, V* p, PcgState* st, double* partials, cudaStream_t s);
// One iteration with the iterate update deferred into the direction update
// (x of type X, r, p, q and the operator of type V): SpMV + alpha, residual
// update + beta, then x += alpha p and p = z + beta p in one pass over p.
template <class V, class X>
void cg_iteration(const Op7<V>& A, X* x, V* r, V* p, V* q, PcgState* st, double* partials, cudaStream_t s);
// The two pointwise kernels of cg_iteration alone (residual update, then the
// deferred iterate update and the direction update), after a SpMV that set
// alpha in the state.
template <class V, class X>
void cg_vector_updates(const Op7<V>& A, X* x, V* r, V* p, V* q, PcgState* st, double* partials, cudaStream_t s);
// p.q and the step length (alpha, or a stagnation stop) for a SpMV that
// wrote q without reducing p.q (the red-black black pass)
template <class V>
void pq_alpha(const Op7<V>& A, const V* p, const V* q, PcgState* st, double* partials, cudaStream_t s);
// Occupancy queries that size cg_iteration's grids: call once per (V, X)
// before the first iteration (outside stream capture).
template <class V, class X> void cg_prepare();
// Largest block count of the cg_iteration kernels on a layout (partial sums).
int cg_max_blocks(const Lay& L);

// ---- red-black reduced pressure solve (fs_redblack.cu)
// The pressure operator's FP32 couplings (cell layout L) seen through the
// packed half layout Lh of one colour: slot (h, j, k) holds the red cell at
// i = 2h + ((j+k)&1) and the black cell at i = 2h + ((j+k+1)&1).
struct RbOp {
  const float* ax;
  const float* ay;
  const float* az;
  Lay L;                  // cell layout of the couplings
  Lay Lh;                 // packed layout of the colour vectors
  const double* extra0;   // deflation term of the first (red) cell
};
Lay make_half_lay(const Lay& L);
int rb_blocks(const Lay& Lh);
// One CG iteration on the black Schur complement: red stage (tau), black
// stage (q = S p, p.q, alpha), then cg_vector_updates on the packed black
// vectors with Ah (layout Lh, dinv16 the packed black bf16 1/diag).
void rb_iteration(const RbOp& A, const Op7<float>& Ah, double* xh, float* rh, float* ph, float* qh, float* tau,
                  PcgState* st, double* partials, cudaStream_t s);
// p64 <- black cells from the packed iterate xh, red cells eliminated in FP64
// from phi and b (the red rows of b - A p64 vanish)
template <class T>
void rb_commit(const T* phi, const double* xh, const double* b, double* p64, const Lay& L, const Lay& Lh, double dx,
               double rho_neg, double rho_pos, int deflate, cudaStream_t s);
// bf16 1/diag(S) of the black Schur complement per packed black slot: the
// black pivots of IC(0) in red-black order
void rb_schur_dinv(const RbOp& A, unsigned short* dinv, cudaStream_t s);
// packed black slots <- black cells of a cell-layout field
template <class S, class D> void rb_gather(const S* full, D* half, const Lay& L, const Lay& Lh, cudaStream_t s);

template <class V, class R = V>
void pcg_resume(const Op7<V>& A, const R* r, V* p, PcgState* st, double* partials, int restart, cudaStream_t s);
int pcg_blocks(const Lay& L);

// ---- projection family (fs_projection.cu)
struct ProjParams {
  double dx, dt, rho_neg, rho_pos;
  int faithful;
};
template <class T>
void divergence_rhs(const T* u, const T* v, const T* w, const Lay& Lc, const Lay& Lu, const Lay& Lv, const Lay& Lw,
                    double dx, double dt, double* b, double* div_out, double* partials, unsigned int* ticket,
                    double* scalars, cudaStream_t s);
// pipe: only the unknowns (cells inside the pipe) count and change
void subtract_mean(double* b, const Lay& Lc, const double* scalars, double* partials, unsigned int* ticket,
                   double* scalars_out, cudaStream_t s, const PipeGeom* pipe = nullptr);
template <class T, class V>
// deflate: the reference's fix of the first cell (the betas of its bottom and
// down Neumann ghosts added to its diagonal, POISSON_SOLVER_3D.h:1145-1179),
// which makes the Neumann system nonsingular; without it the system is
// singular and consistent (b has zero mean) and CG solves it as such.
// pipe: couplings only between two cells inside the pipe (the others are
// Neumann cells, no unknowns: zero couplings, diagonal 1); the deflation of
// the faithful system sits on the pipe's first unknown and adds the beta of
// its down neighbour (POISSON_SOLVER_3D.h:1451-1486).
void build_pressure_operator(const T* phi, const Lay& Lc, double dx, double rho_neg, double rho_pos, V* ax, V* ay, V* az,
                             V* diag, double* extra0, int deflate, cudaStream_t s, unsigned short* dinv16 = nullptr,
                             const PipeGeom* pipe = nullptr);
template <class T>
void defect_residual(const T* phi, const double* p64, const float* x32, const double* b, double* r64, float* r32,
                     const Lay& Lc, double dx, double rho_neg, double rho_pos, double* partials, unsigned int* ticket,
                     double* rr_out, int deflate, cudaStream_t s, const PipeGeom* pipe = nullptr);
void add_correction(double* p64, const float* e, const Lay& Lc, cudaStream_t s);
template <class T>
void velocity_correct(T* f, const T* base, const double* p, const T* phi, const Lay& Lf, const Lay& Lc, int axis,
                      double dx, double dt, double rho_neg, double rho_pos, int faithful, double c0, double c1,
                      const double* kappa, double sigma, cudaStream_t s);
// mean curvature of phi (ghosts must be filled) and max |kappa| near the interface
template <class T>
void curvature(const T* phi, double* kappa, const Lay& L, double dx, int typo, double* kmax, cudaStream_t s);
// ghost-fluid jump terms of the pressure right-hand side (arms to interior
// cells; the reference's wall arms never cross the interface, and `walls` is
// kept for the call sites only); sum(b) of the result lands in sum_out;
// pipe: only the unknowns (cells inside the pipe) get terms and count
template <class T>
void jump_rhs(const T* phi, const double* kappa, double sigma, double* b, const Lay& Lc, double dx, double rho_neg,
              double rho_pos, int walls, double* partials, unsigned int* ticket, double* sum_out, cudaStream_t s,
              const PipeGeom* pipe = nullptr);
template <class T>
void divergence_norms(const T* u, const T* v, const T* w, const Lay& Lc, const Lay& Lu, const Lay& Lv, const Lay& Lw,
                      double dx, double* partials, unsigned int* ticket, double* out2, cudaStream_t s);
template <class T>
void absmax3(const T* u, const T* v, const T* w, const Lay& Lu, const Lay& Lv, const Lay& Lw, double* out3,
             cudaStream_t s);
template <class S, class D> void convert_copy(D* dst, const S* src, const Lay& L, cudaStream_t s);
template <class T> void pack_to_double(double* dst, const T* src, const Lay& L, cudaStream_t s);
template <class T> void unpack_from_double(T* dst, const double* src, const Lay& L, cudaStream_t s);

// ---- viscosity family (fs_viscosity.cu)
// the system of component `axis` from fields of type T, stored in type V
template <class T, class V = T>
void viscosity_system(const T* phi, const T* u, const T* v, const T* w, const Lay& Lc, const Lay& Lu, const Lay& Lv,
                      const Lay& Lw, int axis, double dx, double dt, double rho_neg, double rho_pos, double mu_neg,
                      double mu_pos, V* ax, V* ay, V* az, V* diag, V* rhs, cudaStream_t s);

// The reference's explicit air/water viscosity (VISCOSITY_3D.h:452-563).
// in_place = 0: (ua, va, wa) <- the update of (u, v, w) (the caller swaps);
// in_place = 1: u, v, w updated in place in the reference's order.  Returns
// the number of kernels launched.
template <class T>
int viscosity_explicit(const T* phi, T* u, T* v, T* w, T* ua, T* va, T* wa, const Lay& Lc, const Lay& Lu,
                       const Lay& Lv, const Lay& Lw, double dx, double dt, double rho_neg, double rho_pos,
                       double mu_neg, double mu_pos, int in_place, cudaStream_t s);

// ---- adjoint family (fs_adjoint.cu): primal fields of the storage type T
// (FP64 or FP32), bars FP64; all add into the bars
template <class T>
void adj_weno_levelset(const T* src, const T* u, const T* v, const T* w, const double* out_bar, double* src_bar,
                       double* u_bar, double* v_bar, double* w_bar, const Lay& L, const Lay& Lu, const Lay& Lv,
                       const Lay& Lw, double dx, double eps, double dt, double c1, cudaStream_t s);
void adj_extrap(double* bar, const Lay& L, cudaStream_t s);
template <class T>
void adj_weno_mac(const T* comp, const T* u, const T* v, const T* w, const double* out_bar, double* comp_bar,
                  double* u_bar, double* v_bar, double* w_bar, const Lay& Lc, const Lay& Lu, const Lay& Lv,
                  const Lay& Lw, int axis, double dx, double eps, double dt, cudaStream_t s);
template <class T>
void adj_sussman(const T* src, const T* sgn, const double* out_bar, double* src_bar, double* sgn_bar, const Lay& L,
                 double dx, double eps, double dtau, double c1, int typo, cudaStream_t s);
template <class T>
void adj_sign(const T* phi, const double* sgn_bar, double* phi_bar, const Lay& L, double dx, cudaStream_t s);
template <class T>
void adj_velcorr(const double* p, const T* phi, const double* out_bar, double* in_bar, double* p_bar, double* phi_bar,
                 double* rho_bar, const Lay& Lf, const Lay& Lc, int axis, double dx, double dt, double rn, double rp,
                 double c1, cudaStream_t s);
void adj_divergence(const double* lam, const double* sum_lam, double* in_bar, const Lay& Lf, const Lay& Lc, int axis,
                    double dx, double dt, cudaStream_t s);
void adj_sum(const double* f, const Lay& L, double* partials, unsigned int* ticket, double* out, cudaStream_t s);
template <class T>
void adj_pressure_operator(const T* phi, const double* lam, const double* p, double* phi_bar, double* rho_bar,
                           const Lay& Lc, double dx, double rn, double rp, int deflate, cudaStream_t s);
template <class T>
void adj_visc(const T* phi, const T* ug, const T* vg, const T* wg, const T* x, const double* lam, double* u_bar,
              double* v_bar, double* w_bar, double* phi_bar, double* rho_bar, const Lay& Lc, const Lay& Lu,
              const Lay& Lv, const Lay& Lw, int axis, double dx, double dt, double rn, double rp, double mn,
              double mp, cudaStream_t s);
void adj_zero_walls(double* f, const Lay& L, int axis, cudaStream_t s);
void adj_axpy(double* out, const double* x, double a, const Lay& L, cudaStream_t s);

}  // namespace fsb
