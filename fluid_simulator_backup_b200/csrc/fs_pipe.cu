// Oil/water vertical pipe mode: the geometry kernels of the level-set path
// and the dimensionless body force.
//
// The reference's production scenario (oil_water_simulation with
// PIPE_OPTIONS.is_vertical) is core-annular flow in a pipe along y: a box of
// cells around a cylinder of radius a (in units of the core radius R1),
// periodic along the pipe.  Here the cylinder stays implicit: every kernel
// evaluates the wall distance sqrt(x^2 + z^2) - a of its own point from the
// index (pipe_wall_distance, with the reference's grid positions and
// rounding), so no boundary field is stored or streamed.
//
//   fill_periodic_y           FIELD_STRUCTURE_3D::FillGhostCellsPeriodicInYDirection (scalar,
//                             FIELD_STRUCTURE_3D.h:1328-1431)
//   pipe_levelset_velocities  ADVECTION_3D::SetupBoundaryConditionForVelocity for the level-set
//                             advection (ADVECTION_3D.h:380-490) with the masked periodic fill of
//                             FIELD_STRUCTURE_3D.h:1432-1540
//   pipe_forcing              the vertical branch of EULERIAN_FLUID_SOLVER_3D::ApplyGravity
//                             (EULERIAN_FLUID_SOLVER_3D.h:2276-2326)
//   pipe_velocity_copies      ADVECTION_3D::SetupBoundaryConditionForVelocity for the velocity
//                             advection (ADVECTION_3D.h:551-700): the masked periodic copies with
//                             their linear wall extrapolation, and the guarded copies the ENO3
//                             stencils read along x and z
#include "fs_kernels.h"

namespace fsb {

namespace {

constexpr double kPi = 3.14159265358979323846;  // the reference's PI (MACROS.h:13)

// Ghost shell of a cell field: the y ghosts of interior columns take the
// periodic image (cell 0 and cell ny-1 are the same point, so ghost -m is
// cell ny-1-m and ghost ny-1+m is cell m); the x and z ghost layers, which
// the reference's ghost copy never fills in a vertical pipe, are 0.
template <class T>
__global__ void k_fill_periodic_y(T* f, Lay L) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x - GH;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - GH;
  const int k = blockIdx.z * blockDim.z + threadIdx.z - GH;
  if (i >= L.nx + GH || j >= L.ny + GH || k >= L.nz + GH) return;
  const bool ix = i >= 0 && i < L.nx, jy = j >= 0 && j < L.ny, kz = k >= 0 && k < L.nz;
  if (ix && jy && kz) return;  // interior
  T val = T(0);
  if (ix && kz) val = f[L.at(i, j < 0 ? L.ny - 1 + j : j - L.ny + 1, k)];
  f[L.at(i, j, k)] = val;
}

// The ghost copy the WENO5 update reads, for one face component of a
// vertical pipe, and the zeroing of u and w outside it.  Per face (i,j,k)
// with wall distance b:
//  - the copy is the velocity where b < 1e-8, else 0;
//  - y faces: rows 0 and ny are rewritten with their periodic images (face 0
//    is face ny-1, face ny is face 1) where b < 1e-8;
//  - x (z) faces outside the pipe: 0 when all four transverse neighbours are
//    outside, and the value extrapolated across the wall,
//    (theta - 1)/theta u_in, theta = |b_in|/(|b_in| + |b|), from an inside
//    neighbour along x (z), the + side last; neighbours beyond the face
//    grid have b = 0 (the reference's unfilled ghost layer);
//  - u (w) itself becomes 0 outside the pipe.
// Each face reads only inside faces' velocities, which no thread zeroes, so
// the zeroing in place is race free.
template <class T, int AXIS>
__global__ void k_pipe_ghost_velocity(T* vel, T* ghost, Lay Lf, PipeGeom G) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= Lf.nx || j >= Lf.ny || k >= Lf.nz) return;
  const int g = 1 + AXIS;
  const int64_t f = Lf.at(i, j, k);
  const double b = pipe_wall_distance(G, g, i, k);
  const T v0 = vel[f];
  double out = b < 1e-8 ? (double)v0 : 0.0;
  if (AXIS == 1 && b < 1e-8) {
    if (j == 0) out = (double)vel[Lf.at(i, Lf.ny - 2, k)];
    if (j == Lf.ny - 1) out = (double)vel[Lf.at(i, 1, k)];
  }
  if (AXIS != 1 && b > 0.0) {
    auto bd = [&](int ii, int kk) -> double {
      return (ii < 0 || ii >= Lf.nx || kk < 0 || kk >= Lf.nz) ? 0.0 : pipe_wall_distance(G, g, ii, kk);
    };
    if (bd(i - 1, k) > 0.0 && bd(i + 1, k) > 0.0 && bd(i, k - 1) > 0.0 && bd(i, k + 1) > 0.0) out = 0.0;
    for (int s = -1; s <= 1; s += 2) {
      const int ii = AXIS == 0 ? i + s : i, kk = AXIS == 0 ? k : k + s;
      const double bn = bd(ii, kk);
      if (bn < 0.0) {
        const double theta = fabs(bn) / (fabs(bn) + fabs(b));
        out = (theta - 1.0) / theta * (double)vel[Lf.at(ii, j, kk)];
      }
    }
    vel[f] = T(0);
  }
  ghost[f] = (T)out;
}

// v += R1/V0^2 (dt g_y + dt f/(oil_density rho_f)) on the y faces inside the
// pipe, rho_f = 1 + (eta - 1) H(phi_f), phi_f the mean of the two cells'
// level sets (periodic ghosts filled), H the smeared Heaviside with
// epsilon = 1.5 dy; the centre-line faces (ci, ck) are held fixed.
template <class T>
__global__ void k_pipe_forcing(T* v, const T* __restrict__ phi, Lay Lv, Lay Lc, PipeGeom G, double coef, double gdt,
                               double fdt, double oil, double eta, double eps, double ooe, double oop, int ci,
                               int ck) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= Lv.nx || j >= Lv.ny || k >= Lv.nz) return;
  if (i == ci && k == ck) return;
  if (!(pipe_wall_distance(G, 2, i, k) < 0.0)) return;
  const double pf = 0.5 * ((double)phi[Lc.at(i, j, k)] + (double)phi[Lc.at(i, j - 1, k)]);
  double h;
  if (pf < -eps) h = 0.0;
  else if (pf > eps) h = 1.0;
  else h = (0.5 + pf * ooe * 0.5) + 0.5 * oop * sin(kPi * pf * ooe);
  const double rho = 1.0 + (eta - 1.0) * h;
  const int64_t f = Lv.at(i, j, k);
  v[f] = (T)((double)v[f] + coef * (gdt + 1.0 / (oil * rho) * fdt));
}

// ---- the ghost copies of the pipe's velocity advection

// The masked periodic copy of one face component (FIELD_STRUCTURE_3D.h:
// 1432-1540), over the whole ghosted block: the face's velocity where its
// wall distance b < 1e-8, else 0; for the y component rows 0 and ny take
// their periodic images (face 0 is face ny-1, face ny is face 1) where
// b < 1e-8; the y ghost rows of interior columns take the periodic images
// (the reference's test of b there reads its unfilled ghost rows, 0); the x
// and z ghost layers 0 until the wall extrapolation below.
template <class T, int AXIS>
__global__ void k_pipe_copy(const T* __restrict__ c, T* __restrict__ out, Lay Lf, PipeGeom G) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x - GH;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - GH;
  const int k = blockIdx.z * blockDim.z + threadIdx.z - GH;
  if (i >= Lf.nx + GH || j >= Lf.ny + GH || k >= Lf.nz + GH) return;
  const bool ix = i >= 0 && i < Lf.nx, jy = j >= 0 && j < Lf.ny, kz = k >= 0 && k < Lf.nz;
  const int Ny = Lf.ny;
  double val = 0.0;
  if (ix && kz) {
    if (jy) {
      const bool in = pipe_wall_distance(G, 1 + AXIS, i, k) < 1e-8;
      if (in) {
        int js = j;
        if (AXIS == 1 && j == 0) js = Ny - 2;
        if (AXIS == 1 && j == Ny - 1) js = 1;
        val = (double)c[Lf.at(i, js, k)];
      }
    } else if (AXIS == 1) {
      val = (double)c[Lf.at(i, j < 0 ? Ny - 2 + j : j - Ny + 2, k)];
    } else {
      val = (double)c[Lf.at(i, j < 0 ? Ny - 1 + j : j - Ny + 1, k)];
    }
  }
  out[Lf.at(i, j, k)] = (T)val;
}

// wall distance on the face grid of component AXIS; 0 beyond the grid
// (the reference's unfilled ghost layer of its boundary array)
template <int AXIS>
__device__ __forceinline__ double face_b(const PipeGeom& G, const Lay& Lf, int i, int k) {
  return (i < 0 || i >= Lf.nx || k < 0 || k >= Lf.nz) ? 0.0 : pipe_wall_distance(G, 1 + AXIS, i, k);
}

// The linear wall extrapolation of the masked copy (FIELD_STRUCTURE_3D.h:
// 1563-1610): along each x row (one thread per row) every face from the
// first one outside the pipe to the end of the row, ghost layers included,
// takes 2 c(t-1) - c(t-2) of the velocity itself (right side), then
// 2 c(t+1) - c(t+2) on the left side.  The velocity's own ghost layers are 0.
template <class T, int AXIS>
__global__ void k_pipe_extrap_x(const T* __restrict__ c, T* __restrict__ out, Lay Lf, PipeGeom G) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
  if (j >= Lf.ny || k >= Lf.nz) return;
  const int n = Lf.nx;
  auto cv = [&](int t) { return (double)c[Lf.at(t, j, k)]; };
  for (int i = 0; i < n; ++i)
    if (face_b<AXIS>(G, Lf, i - 1, k) < 0.0 && face_b<AXIS>(G, Lf, i, k) > 0.0)
      for (int t = i; t <= n - 1 + GH; ++t) out[Lf.at(t, j, k)] = (T)(2.0 * cv(t - 1) - cv(t - 2));
  for (int i = 0; i < n; ++i)
    if (face_b<AXIS>(G, Lf, i + 1, k) < 0.0 && face_b<AXIS>(G, Lf, i, k) > 0.0)
      for (int t = i; t >= -GH; --t) out[Lf.at(t, j, k)] = (T)(2.0 * cv(t + 1) - cv(t + 2));
}

// The same along z (one thread per column), after the x rows: it overwrites.
template <class T, int AXIS>
__global__ void k_pipe_extrap_z(const T* __restrict__ c, T* __restrict__ out, Lay Lf, PipeGeom G) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= Lf.nx || j >= Lf.ny) return;
  const int n = Lf.nz;
  auto cv = [&](int t) { return (double)c[Lf.at(i, j, t)]; };
  for (int k = 0; k < n; ++k)
    if (face_b<AXIS>(G, Lf, i, k - 1) < 0.0 && face_b<AXIS>(G, Lf, i, k) > 0.0)
      for (int t = k; t <= n - 1 + GH; ++t) out[Lf.at(i, j, t)] = (T)(2.0 * cv(t - 1) - cv(t - 2));
  for (int k = 0; k < n; ++k)
    if (face_b<AXIS>(G, Lf, i, k + 1) < 0.0 && face_b<AXIS>(G, Lf, i, k) > 0.0)
      for (int t = k; t >= -GH; --t) out[Lf.at(i, j, t)] = (T)(2.0 * cv(t + 1) - cv(t + 2));
}

// The guarded copy the ENO3 reads along x (ALONG = 0) or z (ALONG = 2)
// (ADVECTION_3D.h:560-700): next to each inside face whose neighbour along
// the axis is outside, that neighbour gets (theta-1)/theta times the inside
// face's value, theta = |b_in|/(|b_in| + |b_out|), and the next three faces
// (10t)^t for t = 2, 3, 4, so that no ENO3 stencil choice leaves the pipe.
// One thread per row (x) or column (z), faces in increasing order, the +
// side before the - side, as the reference's loop; writes beyond the
// ghosted block are skipped (the three-cell margin of the pipe keeps them
// inside).
template <class T, int AXIS, int ALONG>
__global__ void k_pipe_guard(const T* __restrict__ gen, T* __restrict__ out, Lay Lf, PipeGeom G) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  const int n = ALONG == 0 ? Lf.nx : Lf.nz;      // along the axis
  const int m = ALONG == 0 ? Lf.nz : Lf.nx;      // the other transverse index
  if (a >= m || j >= Lf.ny) return;
  auto at = [&](int p) { return ALONG == 0 ? Lf.at(p, j, a) : Lf.at(a, j, p); };
  auto bd = [&](int p) { return ALONG == 0 ? face_b<AXIS>(G, Lf, p, a) : face_b<AXIS>(G, Lf, a, p); };
  for (int p = 0; p < n; ++p) {
    const double b = bd(p);
    if (!(b < 0.0)) continue;
    for (int s = 1; s >= -1; s -= 2) {
      const double bn = bd(p + s);
      if (!(bn > 0.0)) continue;
      const double theta = fabs(b) / (fabs(bn) + fabs(b));
      out[at(p + s)] = (T)((theta - 1.0) / theta * (double)gen[at(p)]);
      for (int t = 2; t <= 4; ++t) {
        const int q = p + s * t;
        if (q < -GH || q > n - 1 + GH) continue;
        out[at(q)] = (T)(t == 2 ? 400.0 : t == 3 ? 27000.0 : 2560000.0);  // (10 t)^t
      }
    }
  }
}

template <class T, int AXIS>
void pipe_copies_axis(const T* c, T* gen, T* gx, T* gz, const Lay& Lf, const PipeGeom& G, cudaStream_t s) {
  const dim3 b(32, 4, 2);
  const dim3 g((Lf.nx + 2 * GH + 31) / 32, (Lf.ny + 2 * GH + 3) / 4, (Lf.nz + 2 * GH + 1) / 2);
  k_pipe_copy<T, AXIS><<<g, b, 0, s>>>(c, gen, Lf, G);
  k_pipe_extrap_x<T, AXIS><<<dim3((Lf.ny + 63) / 64, Lf.nz), 64, 0, s>>>(c, gen, Lf, G);
  k_pipe_extrap_z<T, AXIS><<<dim3((Lf.nx + 63) / 64, Lf.ny), 64, 0, s>>>(c, gen, Lf, G);
  const size_t bytes = (size_t)Lf.total * sizeof(T);
  cudaMemcpyAsync(gx, gen, bytes, cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(gz, gen, bytes, cudaMemcpyDeviceToDevice, s);
  k_pipe_guard<T, AXIS, 0><<<dim3((Lf.nz + 63) / 64, Lf.ny), 64, 0, s>>>(gen, gx, Lf, G);
  k_pipe_guard<T, AXIS, 2><<<dim3((Lf.nx + 63) / 64, Lf.ny), 64, 0, s>>>(gen, gz, Lf, G);
}

}  // namespace

template <class T>
int pipe_velocity_copies(const T* const comp[3], T* const gen[3], T* const gx[3], T* const gz[3], const Lay* const L[3],
                         const PipeGeom& G, cudaStream_t s) {
  pipe_copies_axis<T, 0>(comp[0], gen[0], gx[0], gz[0], *L[0], G, s);
  pipe_copies_axis<T, 1>(comp[1], gen[1], gx[1], gz[1], *L[1], G, s);
  pipe_copies_axis<T, 2>(comp[2], gen[2], gx[2], gz[2], *L[2], G, s);
  return 15;  // kernels launched
}

template <class T>
void fill_periodic_y(T* f, const Lay& L, cudaStream_t s) {
  const dim3 b(32, 4, 2);
  const dim3 g((L.nx + 2 * GH + 31) / 32, (L.ny + 2 * GH + 3) / 4, (L.nz + 2 * GH + 1) / 2);
  k_fill_periodic_y<T><<<g, b, 0, s>>>(f, L);
}

template <class T>
void pipe_levelset_velocities(T* u, T* v, T* w, T* ug, T* vg, T* wg, const Lay& Lu, const Lay& Lv, const Lay& Lw,
                              const PipeGeom& G, cudaStream_t s) {
  Launch3 a = launch3(Lu.nx, Lu.ny, Lu.nz), b = launch3(Lv.nx, Lv.ny, Lv.nz), c = launch3(Lw.nx, Lw.ny, Lw.nz);
  k_pipe_ghost_velocity<T, 0><<<a.grid, a.block, 0, s>>>(u, ug, Lu, G);
  k_pipe_ghost_velocity<T, 1><<<b.grid, b.block, 0, s>>>(v, vg, Lv, G);
  k_pipe_ghost_velocity<T, 2><<<c.grid, c.block, 0, s>>>(w, wg, Lw, G);
}

template <class T>
void pipe_forcing(T* v, const T* phi, const Lay& Lv, const Lay& Lc, const PipeGeom& G, double coef, double gdt,
                  double fdt, double oil_density, double eta, double eps, cudaStream_t s) {
  Launch3 a = launch3(Lv.nx, Lv.ny, Lv.nz);
  k_pipe_forcing<T><<<a.grid, a.block, 0, s>>>(v, phi, Lv, Lc, G, coef, gdt, fdt, oil_density, eta, eps, 1.0 / eps,
                                                1.0 / kPi, (Lc.nx - 1) / 2, (Lc.nz - 1) / 2);
}

// ---- the pipe's projection (PROJECTION_3D.h:681-744, 1099-1449, 1519-1610)

// The velocity of face (i, j, k) as the pipe's divergence reads it
// (SetupBoundaryConditionsForVelocityDivergence, PROJECTION_3D.h:1519-1610):
// x and z faces outside the pipe (b > 0) take 0 when all four transverse
// neighbours are outside, else the linear extrapolation across the wall,
// (theta - 1)/theta times the inside neighbour along the axis, the - side
// first, theta = |b_in|/(|b_in| + |b|) (neighbours beyond the face grid have
// b = 0, the boundary array's unfilled ghost layer); the other faces the
// masked periodic copy: the face's own velocity where b < 1e-8 (for the y
// component face 0 reads face ny-1 and face ny face 1), else 0.
template <class T, int AXIS>
__device__ __forceinline__ double pipe_div_face(const T* __restrict__ vel, const Lay& Lf, const PipeGeom& G, int i,
                                                int j, int k) {
  const int g = 1 + AXIS;
  const double b = pipe_wall_distance(G, g, i, k);
  if (AXIS != 1 && b > 0.0) {
    auto bd = [&](int ii, int kk) -> double {
      return (ii < 0 || ii >= Lf.nx || kk < 0 || kk >= Lf.nz) ? 0.0 : pipe_wall_distance(G, g, ii, kk);
    };
    if (bd(i - 1, k) > 0.0 && bd(i + 1, k) > 0.0 && bd(i, k - 1) > 0.0 && bd(i, k + 1) > 0.0) return 0.0;
    for (int s = -1; s <= 1; s += 2) {
      const int ii = AXIS == 0 ? i + s : i, kk = AXIS == 0 ? k : k + s;
      const double bn = bd(ii, kk);
      if (bn < 0.0) {
        const double theta = fabs(bn) / (fabs(bn) + fabs(b));
        return (theta - 1.0) / theta * (double)vel[Lf.at(ii, j, kk)];
      }
    }
    return 0.0;
  }
  if (b < 1e-8) {
    if (AXIS == 1 && j == 0) return (double)vel[Lf.at(i, Lf.ny - 2, k)];
    if (AXIS == 1 && j == Lf.ny - 1) return (double)vel[Lf.at(i, 1, k)];
    return (double)vel[Lf.at(i, j, k)];
  }
  return 0.0;
}

// b = -(div u)/dt on the cells inside the pipe, 0 on the others (no
// unknowns), and sum(b) for the mean removal (DetermineDivergence,
// PROJECTION_3D.h:697-722: one_over_dx (u_r - u_l) + one_over_dy (v_t - v_b)
// + one_over_dz (w_u - w_d) in that order, then times 1/dt).
template <class T>
__global__ void k_pipe_divergence_rhs(const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ w,
                                      Lay Lc, Lay Lu, Lay Lv, Lay Lw, PipeGeom G, double inv_h, double inv_dt,
                                      double* __restrict__ b, double* __restrict__ div_out, double* partials,
                                      unsigned int* ticket, double* scalars) {
  double bv = 0.0;
  Cursor cur;
  for (cur.init(Lc); cur.valid(Lc); cur.next(Lc)) {
    const int i = cur.i, j = cur.j, k = cur.k;
    const int64_t c = Lc.at(i, j, k);
    if (pipe_solid(G, i, k)) {
      div_out[c] = 0.0;
      b[c] = 0.0;
      continue;
    }
    double d = inv_h * (pipe_div_face<T, 0>(u, Lu, G, i + 1, j, k) - pipe_div_face<T, 0>(u, Lu, G, i, j, k));
    d += inv_h * (pipe_div_face<T, 1>(v, Lv, G, i, j + 1, k) - pipe_div_face<T, 1>(v, Lv, G, i, j, k));
    d += inv_h * (pipe_div_face<T, 2>(w, Lw, G, i, j, k + 1) - pipe_div_face<T, 2>(w, Lw, G, i, j, k));
    const double dv = d * inv_dt;
    div_out[c] = dv;
    b[c] = -dv;
    bv += -dv;
  }
  bv = block_sum(bv);
  double tot;
  if (grid_reduce_sum(bv, partials, ticket, &tot)) scalars[0] = tot;
}

// UpdateVelocityByPressureGradientVariableDensity of a vertical pipe
// (PROJECTION_3D.h:1151-1449), one component.  Face (i, j, k) lies between
// cell c = (i, j, k) and cell n one step back along the axis.  It is updated
// when it is not one of the centre-line faces Solve_Velocity holds fixed,
// c is an unknown (inside the pipe) and n is one too or c is the first
// unknown (its row index 0 makes the reference's bc*bc_n >= 0 hold against
// a Neumann cell, whose pressure the solve never writes); y faces only for
// 0 < j < ny.  Same-phase faces: -= dt (p_c - p_n)/rho_c/h with the sharp
// density of c; faces with phi_c phi_n <= 0: -= dt (p_c - p_n +- gamma)/
// rho_f/h, gamma = (jc_c|phi_n| + jc_n|phi_c|)/(|phi_n| + |phi_c|), jc =
// sigma kappa, + when phi_c <= 0, rho_f = rn + (rp - rn) H(phi_f) with phi_f
// the face average and H the projection's smeared Heaviside of epsilon eps.
template <class T, int AXIS>
__global__ void k_pipe_velocity_correct(T* __restrict__ f, const double* __restrict__ p, const T* __restrict__ phi,
                                        const double* __restrict__ kappa, Lay Lf, Lay Lc, PipeGeom G, double inv_h,
                                        double dt, double rn, double rp, double sigma, double eps, int fi0, int fi1,
                                        int fk0, int fk1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= Lf.nx || j >= Lf.ny || k >= Lf.nz) return;
  if ((i == fi0 || i == fi1) && (k == fk0 || k == fk1)) return;  // the fixed centre line
  if (AXIS == 1 && (j == 0 || j >= Lc.ny)) return;
  if (AXIS == 0 && i >= Lc.nx) return;  // the last face's + cell is the Neumann ghost layer
  if (AXIS == 2 && k >= Lc.nz) return;
  if (pipe_solid(G, i, k)) return;
  const int in = AXIS == 0 ? i - 1 : i, jn = AXIS == 1 ? j - 1 : j, kn = AXIS == 2 ? k - 1 : k;
  const bool first = i == G.fi && j == G.fj && k == G.fk;
  if (in < 0 || kn < 0 || (pipe_solid(G, in, kn) && !first)) return;
  const int64_t c = Lc.at(i, j, k), n = Lc.at(in, jn, kn);
  const double pc = (double)phi[c], pn = (double)phi[n];
  const double dp = p[c] - p[n];
  const int64_t fo = Lf.at(i, j, k);
  double val = (double)f[fo];
  if (pc * pn > 0.0) {
    val -= dt * dp * (1.0 / (pc <= 0.0 ? rn : rp)) * inv_h;
  } else {
    const double jc = sigma * kappa[c], jn = sigma * kappa[n];
    const double ac = fabs(pc), an = fabs(pn);
    const double gamma = (jc * an + jn * ac) / (an + ac);
    const double pf = 0.5 * (pc + pn);
    double h;
    if (pf < -eps) h = 0.0;
    else if (pf > eps) h = 1.0;
    else h = (0.5 + pf * (1.0 / eps) * 0.5) + 0.5 * (1.0 / kPi) * sin(kPi * pf * (1.0 / eps));
    const double inv_rf = 1.0 / (rn + (rp - rn) * h);
    val -= dt * (pc <= 0.0 ? dp + gamma : dp - gamma) * inv_rf * inv_h;
  }
  f[fo] = (T)val;
}

// The periodic rows the pipe's velocity update ends with: u and w row ny-1
// takes row 0; v row ny takes row 1 and row 0 takes row ny-1.
template <class T>
__global__ void k_pipe_periodic_rows(T* u, T* v, T* w, Lay Lu, Lay Lv, Lay Lw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < Lu.nx && k < Lu.nz) u[Lu.at(i, Lu.ny - 1, k)] = u[Lu.at(i, 0, k)];
  if (i < Lv.nx && k < Lv.nz) {
    v[Lv.at(i, Lv.ny - 1, k)] = v[Lv.at(i, 1, k)];
    v[Lv.at(i, 0, k)] = v[Lv.at(i, Lv.ny - 2, k)];
  }
  if (i < Lw.nx && k < Lw.nz) w[Lw.at(i, Lw.ny - 1, k)] = w[Lw.at(i, 0, k)];
}

template <class T>
void pipe_divergence_rhs(const T* u, const T* v, const T* w, const Lay& Lc, const Lay& Lu, const Lay& Lv,
                         const Lay& Lw, const PipeGeom& G, double dx, double dt, double* b, double* div_out,
                         double* partials, unsigned int* ticket, double* scalars, cudaStream_t s) {
  k_pipe_divergence_rhs<T><<<pcg_blocks(Lc), kRedThreads, 0, s>>>(u, v, w, Lc, Lu, Lv, Lw, G, 1.0 / dx, 1.0 / dt, b,
                                                                  div_out, partials, ticket, scalars);
}

template <class T>
void pipe_velocity_correct(T* u, T* v, T* w, const double* p, const T* phi, const double* kappa, const Lay& Lc,
                           const Lay& Lu, const Lay& Lv, const Lay& Lw, const PipeGeom& G, double dx, double dt,
                           double rho_neg, double rho_pos, double sigma, cudaStream_t s) {
  const double eps = 1.5 * dx, inv_h = 1.0 / dx;
  // the faces Solve_Velocity holds fixed (ADVECTION_3D.h:246-275), as eno3_pipe
  const int ci = (Lc.nx - 1) / 2, ck = (Lc.nz - 1) / 2;
  Launch3 a = launch3(Lu.nx, Lu.ny, Lu.nz), b = launch3(Lv.nx, Lv.ny, Lv.nz), c = launch3(Lw.nx, Lw.ny, Lw.nz);
  k_pipe_velocity_correct<T, 0><<<a.grid, a.block, 0, s>>>(u, p, phi, kappa, Lu, Lc, G, inv_h, dt, rho_neg, rho_pos,
                                                           sigma, eps, (Lu.nx - 1) / 2, (Lu.nx - 1) / 2 + 1, ck, ck);
  k_pipe_velocity_correct<T, 1><<<b.grid, b.block, 0, s>>>(v, p, phi, kappa, Lv, Lc, G, inv_h, dt, rho_neg, rho_pos,
                                                           sigma, eps, ci, ci, ck, ck);
  k_pipe_velocity_correct<T, 2><<<c.grid, c.block, 0, s>>>(w, p, phi, kappa, Lw, Lc, G, inv_h, dt, rho_neg, rho_pos,
                                                           sigma, eps, ci, ci, (Lw.nz - 1) / 2, (Lw.nz - 1) / 2 + 1);
  const dim3 rb(32, 4);
  const dim3 rg((Lu.nx + 31) / 32, (Lw.nz + 3) / 4);
  k_pipe_periodic_rows<T><<<rg, rb, 0, s>>>(u, v, w, Lu, Lv, Lw);
}

#define FS_PIPE_INST(T)                                                                                          \
  template void fill_periodic_y<T>(T*, const Lay&, cudaStream_t);                                              \
  template void pipe_levelset_velocities<T>(T*, T*, T*, T*, T*, T*, const Lay&, const Lay&, const Lay&,          \
                                            const PipeGeom&, cudaStream_t);                                     \
  template void pipe_forcing<T>(T*, const T*, const Lay&, const Lay&, const PipeGeom&, double, double, double,  \
                                double, double, double, cudaStream_t);                                          \
  template void pipe_divergence_rhs<T>(const T*, const T*, const T*, const Lay&, const Lay&, const Lay&,         \
                                       const Lay&, const PipeGeom&, double, double, double*, double*, double*,   \
                                       unsigned int*, double*, cudaStream_t);                                    \
  template void pipe_velocity_correct<T>(T*, T*, T*, const double*, const T*, const double*, const Lay&,         \
                                         const Lay&, const Lay&, const Lay&, const PipeGeom&, double, double,    \
                                         double, double, double, cudaStream_t);
#define FS_PIPE_INST2(T)                                                                                         \
  template int pipe_velocity_copies<T>(const T* const[3], T* const[3], T* const[3], T* const[3],                 \
                                       const Lay* const[3], const PipeGeom&, cudaStream_t);
FS_PIPE_INST2(float)
FS_PIPE_INST2(double)
FS_PIPE_INST(float)
FS_PIPE_INST(double)

}  // namespace fsb
