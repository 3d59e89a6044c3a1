// Semi-implicit viscosity (VISCOSITY_3D.h:567-990 with the system of
// POISSON_SOLVER_3D.h:3359-3496), one velocity component at a time.
//
// The reference solves (1 + sum c/dx^2) u_f - sum c_arm/dx^2 u_nb = u* +
// dt/rho_f (transpose stress terms), with c = 2 dt mu/rho_f on the two normal
// arms and dt mu/rho_f on the four tangential arms.  Multiplying each row by
// the face density rho_f gives the symmetric positive definite form
//   (rho_f + sum k dt mu_arm/dx^2) u_f - sum k dt mu_arm/dx^2 u_nb = rho_f*rhs
// (k = 2 on the normal arms) with the same solution, which is what the
// conjugate-gradient engine here solves.  Each arm coupling is computed once
// per arm midpoint, so the matrix is exactly symmetric in floating point.
//
// Box boundary: the wall-normal faces of the component are Dirichlet zero
// (no penetration) and velocity ghosts beyond the walls are zero; both enter
// the diagonal through their arm couplings and drop out of the right-hand
// side.  Wall rows become identity rows with zero right-hand side.
#include "fs_kernels.h"

namespace fsb {

__device__ __forceinline__ double heaviside_visc(double phi, double e) {
  // VISCOSITY_3D.h:1234-1253
  const double ooe = 1.0 / e, oop = 1.0 / 3.14159265358979323846;
  if (phi < -e) return 0.0;
  if (phi > e) return 1.0;
  return 0.5 * ((1.0 + phi * ooe) + oop * sin(3.14159265358979323846 * phi * ooe));
}

template <class T>
struct PhiX {  // phi with a one-layer linear extrapolation across the walls
  const T* phi;
  Lay L;
  __device__ double at(int i, int j, int k) const {
    // clamp-and-extrapolate dimension by dimension (one layer)
    int ii = min(max(i, 0), L.nx - 1), jj = min(max(j, 0), L.ny - 1), kk = min(max(k, 0), L.nz - 1);
    auto val = [&](int a, int b, int c) { return (double)phi[L.at(a, b, c)]; };
    auto ex = [&](int a, int b, int c) -> double {
      // extend in x
      if (i < 0) return 2.0 * val(0, b, c) - val(1, b, c);
      if (i >= L.nx) return 2.0 * val(L.nx - 1, b, c) - val(L.nx - 2, b, c);
      return val(a, b, c);
    };
    auto ey = [&](int a, int b, int c) -> double {
      if (j < 0) return 2.0 * ex(a, 0, c) - ex(a, 1, c);
      if (j >= L.ny) return 2.0 * ex(a, L.ny - 1, c) - ex(a, L.ny - 2, c);
      return ex(a, b, c);
    };
    if (k < 0) return 2.0 * ey(ii, jj, 0) - ey(ii, jj, 1);
    if (k >= L.nz) return 2.0 * ey(ii, jj, L.nz - 1) - ey(ii, jj, L.nz - 2);
    return ey(ii, jj, kk);
  }
};

// Face (i,j,k) of component `axis` sits between cell (i,j,k) and the cell
// one step back along the axis.  Cells around the face are addressed in
// "face coordinates" relative to that low cell.
template <class T>
__global__ void k_visc_system(const T* __restrict__ phi, const T* __restrict__ u, const T* __restrict__ v,
                              const T* __restrict__ w, Lay Lc, Lay Lu, Lay Lv, Lay Lw, Lay Lf, int axis, double inv_h,
                              double dt, double rn, double rp, double mn, double mp, T* __restrict__ ax,
                              T* __restrict__ ay, T* __restrict__ az, T* __restrict__ diag, T* __restrict__ rhs) {
  FS_IJK(Lf);
  const int64_t f = Lf.at(i, j, k);
  const PhiX<T> P{phi, Lc};
  const double e = 1.5 / inv_h;
  const double inv2 = inv_h * inv_h;
  const int ea[3] = {axis == 0, axis == 1, axis == 2};
  // cell on the low side of the face
  const int li = i - ea[0], lj = j - ea[1], lk = k - ea[2];
  auto mu_of = [&](double ph) { return mn + (mp - mn) * heaviside_visc(ph, e); };
  // density at the face from the face-averaged phi
  const double rho_f = rn + (rp - rn) * heaviside_visc(0.5 * (P.at(li, lj, lk) + P.at(i, j, k)), e);
  // coupling on the low arm along direction d (between this face and the
  // face one step back along d): normal arm -> the low cell, tangential arm
  // -> the edge shared by the four cells {low, high} x {d-1, d}
  double mu_low[3], mu_high[3], low[3], high[3];
  for (int d = 0; d < 3; ++d) {
    const int di = d == 0, dj = d == 1, dk = d == 2;
    if (d == axis) {
      mu_low[d] = mu_of(P.at(li, lj, lk));
      mu_high[d] = mu_of(P.at(i, j, k));
    } else {
      // canonical order: (low cell, d-1), (low cell), (high cell, d-1), (high cell)
      const double s_lo = ((P.at(li - di, lj - dj, lk - dk) + P.at(li, lj, lk)) + P.at(i - di, j - dj, k - dk)) +
                          P.at(i, j, k);
      // the edge one step up along d, seen from the next face (same order)
      const double s_hi = ((P.at(li, lj, lk) + P.at(li + di, lj + dj, lk + dk)) + P.at(i, j, k)) +
                          P.at(i + di, j + dj, k + dk);
      mu_low[d] = mu_of(0.25 * s_lo);
      mu_high[d] = mu_of(0.25 * s_hi);
    }
    const double kk = d == axis ? 2.0 : 1.0;
    low[d] = kk * dt * mu_low[d] * inv2;
    high[d] = kk * dt * mu_high[d] * inv2;
  }
  const int e_ax = axis == 0 ? i : (axis == 1 ? j : k);
  const int n_ax = axis == 0 ? Lf.nx : (axis == 1 ? Lf.ny : Lf.nz);
  const bool wall = e_ax == 0 || e_ax == n_ax - 1;
  // couplings stored at this face couple it with the face one step back;
  // couplings that touch a wall face are zeroed (Dirichlet neighbour)
  const bool low_is_wall[3] = {axis == 0 && i == 1, axis == 1 && j == 1, axis == 2 && k == 1};
  ax[f] = (T)((wall || low_is_wall[0] || i == 0) ? 0.0 : low[0]);
  ay[f] = (T)((wall || low_is_wall[1] || j == 0) ? 0.0 : low[1]);
  az[f] = (T)((wall || low_is_wall[2] || k == 0) ? 0.0 : low[2]);
  if (wall) {
    diag[f] = (T)1.0;
    rhs[f] = (T)0.0;
    return;
  }
  diag[f] = (T)(rho_f + ((((low[0] + high[0]) + low[1]) + high[1]) + low[2]) + high[2]);
  // explicit transpose terms (VISCOSITY_3D.h:620-630): for each tangential
  // direction t, d/dt( mu_edge * d(vel_t)/d(axis) ) with zero ghosts
  const T* comp[3] = {u, v, w};
  const Lay lay[3] = {Lu, Lv, Lw};
  double ex = (double)comp[axis][f];
  const double coef = dt / rho_f;
  for (int t = 0; t < 3; ++t) {
    if (t == axis) continue;
    const int ti = t == 0, tj = t == 1, tk = t == 2;
    const T* vt = comp[t];
    const Lay& Lt = lay[t];
    // vel_t at (face coords) + e_t and at the same place shifted back along axis
    const double hi_a = (double)vt[Lt.at(i + ti, j + tj, k + tk)];
    const double hi_b = (double)vt[Lt.at(i + ti - ea[0], j + tj - ea[1], k + tk - ea[2])];
    const double lo_a = (double)vt[Lt.at(i, j, k)];
    const double lo_b = (double)vt[Lt.at(i - ea[0], j - ea[1], k - ea[2])];
    ex = ex + coef * (inv_h * (mu_high[t] * inv_h * (hi_a - hi_b) - mu_low[t] * inv_h * (lo_a - lo_b)));
  }
  rhs[f] = (T)(rho_f * ex);
}

template <class T>
void viscosity_system(const T* phi, const T* u, const T* v, const T* w, const Lay& Lc, const Lay& Lu, const Lay& Lv,
                      const Lay& Lw, int axis, double dx, double dt, double rho_neg, double rho_pos, double mu_neg,
                      double mu_pos, T* ax, T* ay, T* az, T* diag, T* rhs, cudaStream_t s) {
  const Lay& Lf = axis == 0 ? Lu : (axis == 1 ? Lv : Lw);
  Launch3 g = launch3(Lf.nx, Lf.ny, Lf.nz);
  k_visc_system<T><<<g.grid, g.block, 0, s>>>(phi, u, v, w, Lc, Lu, Lv, Lw, Lf, axis, 1.0 / dx, dt, rho_neg, rho_pos,
                                               mu_neg, mu_pos, ax, ay, az, diag, rhs);
}

template void viscosity_system<float>(const float*, const float*, const float*, const float*, const Lay&, const Lay&,
                                      const Lay&, const Lay&, int, double, double, double, double, double, double,
                                      float*, float*, float*, float*, float*, cudaStream_t);
template void viscosity_system<double>(const double*, const double*, const double*, const double*, const Lay&,
                                       const Lay&, const Lay&, const Lay&, int, double, double, double, double, double,
                                       double, double*, double*, double*, double*, double*, cudaStream_t);

}  // namespace fsb
