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

#define FS_PIPE_INST(T)                                                                                          \
  template void fill_periodic_y<T>(T*, const Lay&, cudaStream_t);                                              \
  template void pipe_levelset_velocities<T>(T*, T*, T*, T*, T*, T*, const Lay&, const Lay&, const Lay&,          \
                                            const PipeGeom&, cudaStream_t);                                     \
  template void pipe_forcing<T>(T*, const T*, const Lay&, const Lay&, const PipeGeom&, double, double, double,  \
                                double, double, double, cudaStream_t);
#define FS_PIPE_INST2(T)                                                                                         \
  template int pipe_velocity_copies<T>(const T* const[3], T* const[3], T* const[3], T* const[3],                 \
                                       const Lay* const[3], const PipeGeom&, cudaStream_t);
FS_PIPE_INST2(float)
FS_PIPE_INST2(double)
FS_PIPE_INST(float)
FS_PIPE_INST(double)

}  // namespace fsb
