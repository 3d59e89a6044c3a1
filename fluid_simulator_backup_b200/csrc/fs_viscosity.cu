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
// The component's axis is a template parameter so that every per-direction
// array below is indexed by compile-time constants (registers, no stack).
template <class T, class V, int axis>
__global__ void k_visc_system(const T* __restrict__ phi, const T* __restrict__ u, const T* __restrict__ v,
                              const T* __restrict__ w, Lay Lc, Lay Lu, Lay Lv, Lay Lw, Lay Lf, double inv_h,
                              double dt, double rn, double rp, double mn, double mp, V* __restrict__ ax,
                              V* __restrict__ ay, V* __restrict__ az, V* __restrict__ diag, V* __restrict__ rhs) {
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
#pragma unroll
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
  ax[f] = (V)((wall || low_is_wall[0] || i == 0) ? 0.0 : low[0]);
  ay[f] = (V)((wall || low_is_wall[1] || j == 0) ? 0.0 : low[1]);
  az[f] = (V)((wall || low_is_wall[2] || k == 0) ? 0.0 : low[2]);
  if (wall) {
    diag[f] = (V)1.0;
    rhs[f] = (V)0.0;
    return;
  }
  diag[f] = (V)(rho_f + ((((low[0] + high[0]) + low[1]) + high[1]) + low[2]) + high[2]);
  // explicit transpose terms (VISCOSITY_3D.h:620-630): for each tangential
  // direction t, d/dt( mu_edge * d(vel_t)/d(axis) ) with zero ghosts
  const T* own = axis == 0 ? u : (axis == 1 ? v : w);
  double ex = (double)own[f];
  const double coef = dt / rho_f;
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    if (t == axis) continue;
    const int ti = t == 0, tj = t == 1, tk = t == 2;
    const T* vt = t == 0 ? u : (t == 1 ? v : w);
    const Lay& Lt = t == 0 ? Lu : (t == 1 ? Lv : Lw);
    // vel_t at (face coords) + e_t and at the same place shifted back along axis
    const double hi_a = (double)vt[Lt.at(i + ti, j + tj, k + tk)];
    const double hi_b = (double)vt[Lt.at(i + ti - ea[0], j + tj - ea[1], k + tk - ea[2])];
    const double lo_a = (double)vt[Lt.at(i, j, k)];
    const double lo_b = (double)vt[Lt.at(i - ea[0], j - ea[1], k - ea[2])];
    ex = ex + coef * (inv_h * (mu_high[t] * inv_h * (hi_a - hi_b) - mu_low[t] * inv_h * (lo_a - lo_b)));
  }
  rhs[f] = (V)(rho_f * ex);
}

// ---------------------------------------------------------------------------
// The reference's air/water viscosity: the explicit variable-viscosity stress
// update of VISCOSITY_3D::ApplyViscosity (VISCOSITY_3D.h:452-563).  Per face
// of component a: the smeared density of the face-averaged phi, the smeared
// viscosity at the two cells across the face (normal stress, factor 2) and
// at the four edge averages (shear), each sample summed in the reference's
// operand order (VISCOSITY_3D.h:462-470, 502-510, 541-549).
//
// corrected (default): one explicit Euler step of the stress divergence from
// the input velocities into separate output arrays, every transposed-stress
// term on its own edge, wall-normal faces unchanged.  in_place
// (FS_FLAG_VISCOSITY_IN_PLACE): as the reference runs on one thread - x,
// then y, then z, each updated in place in (k, j, i) order, wall faces
// included, with the reference's velocity indices (its y update reads w one
// level low on both z edges, its z update reads u and v on the low edge's
// column/row for the high edge too).  The in-place order is reproduced by
// hyperplanes i + j + k = s: a face depends on its own component only through
// its x-1, y-1, z-1 neighbours (hyperplane s-1, already updated) and x+1,
// y+1, z+1 neighbours (s+1, not yet), so one launch per hyperplane reads
// exactly what the sequential loop reads.
// ---------------------------------------------------------------------------

struct ExplicitViscosity {
  Lay Lc, Lu, Lv, Lw;
  int axis;
  double inv_h, dt, rn, rp, mn, mp;
};

template <class T, bool IN_PLACE>
__device__ __forceinline__ double explicit_visc_face(const ExplicitViscosity& X, const PhiX<T>& P, const T* u,
                                                     const T* v, const T* w, int i, int j, int k) {
  const double e = 1.5 / X.inv_h, inv = X.inv_h;
  auto ph = [&](int di, int dj, int dk) { return P.at(i + di, j + dj, k + dk); };
  double half, hi, lo, e1, e2, e3, e4;
  if (X.axis == 0) {
    half = 0.5 * (ph(-1, 0, 0) + ph(0, 0, 0));
    hi = ph(0, 0, 0);
    lo = ph(-1, 0, 0);
    e1 = 0.25 * (((ph(-1, 0, 0) + ph(0, 0, 0)) + ph(-1, 1, 0)) + ph(0, 1, 0));
    e2 = 0.25 * (((ph(-1, 0, 0) + ph(0, 0, 0)) + ph(-1, -1, 0)) + ph(0, -1, 0));
    e3 = 0.25 * (((ph(-1, 0, 0) + ph(0, 0, 0)) + ph(-1, 0, 1)) + ph(0, 0, 1));
    e4 = 0.25 * (((ph(-1, 0, 0) + ph(0, 0, 0)) + ph(-1, 0, -1)) + ph(0, 0, -1));
  } else if (X.axis == 1) {
    half = 0.5 * (ph(0, -1, 0) + ph(0, 0, 0));
    hi = ph(0, 0, 0);
    lo = ph(0, -1, 0);
    e1 = 0.25 * (((ph(0, -1, 0) + ph(1, -1, 0)) + ph(0, 0, 0)) + ph(1, 0, 0));
    e2 = 0.25 * (((ph(-1, -1, 0) + ph(0, -1, 0)) + ph(-1, 0, 0)) + ph(0, 0, 0));
    e3 = 0.25 * (((ph(0, -1, 1) + ph(0, -1, 0)) + ph(0, 0, 1)) + ph(0, 0, 0));
    e4 = 0.25 * (((ph(0, -1, -1) + ph(0, -1, 0)) + ph(0, 0, -1)) + ph(0, 0, 0));
  } else {
    half = 0.5 * (ph(0, 0, -1) + ph(0, 0, 0));
    hi = ph(0, 0, 0);
    lo = ph(0, 0, -1);
    e1 = 0.25 * (((ph(0, 0, -1) + ph(1, 0, -1)) + ph(0, 0, 0)) + ph(1, 0, 0));
    e2 = 0.25 * (((ph(0, 0, -1) + ph(-1, 0, -1)) + ph(0, 0, 0)) + ph(-1, 0, 0));
    e3 = 0.25 * (((ph(0, 0, -1) + ph(0, 1, -1)) + ph(0, 0, 0)) + ph(0, 1, 0));
    e4 = 0.25 * (((ph(0, 0, -1) + ph(0, -1, -1)) + ph(0, 0, 0)) + ph(0, -1, 0));
  }
  auto mu = [&](double p) { return X.mn + (X.mp - X.mn) * heaviside_visc(p, e); };
  const double rho_h = X.rn + (X.rp - X.rn) * heaviside_visc(half, e);
  const double m0 = mu(hi), m1 = mu(lo), m2 = mu(e1), m3 = mu(e2), m4 = mu(e3), m5 = mu(e4);
  const T* comp[3] = {u, v, w};
  const Lay lay[3] = {X.Lu, X.Lv, X.Lw};
  auto at = [&](int c, int di, int dj, int dk) { return (double)comp[c][lay[c].at(i + di, j + dj, k + dk)]; };
  const double coef = X.dt * (1.0 / rho_h);
  if (X.axis == 0) {
    const double uc = at(0, 0, 0, 0);
    const double first = 2.0 * coef * inv * (m0 * inv * (at(0, 1, 0, 0) - uc) - m1 * inv * (uc - at(0, -1, 0, 0)));
    const double second = coef * inv * (m2 * (inv * (at(0, 0, 1, 0) - uc) + inv * (at(1, 0, 1, 0) - at(1, -1, 1, 0))) -
                                        m3 * (inv * (uc - at(0, 0, -1, 0)) + inv * (at(1, 0, 0, 0) - at(1, -1, 0, 0))));
    const double third = coef * inv * (m4 * (inv * (at(0, 0, 0, 1) - uc) + inv * (at(2, 0, 0, 1) - at(2, -1, 0, 1))) -
                                       m5 * (inv * (uc - at(0, 0, 0, -1)) + inv * (at(2, 0, 0, 0) - at(2, -1, 0, 0))));
    return uc + ((first + second) + third);
  }
  if (X.axis == 1) {
    const double vc = at(1, 0, 0, 0);
    const int zt = IN_PLACE ? 0 : 1;  // the w level of the z+ edge
    const double first = coef * inv * (m2 * (inv * (at(0, 1, 0, 0) - at(0, 1, -1, 0)) + inv * (at(1, 1, 0, 0) - vc)) -
                                       m3 * (inv * (at(0, 0, 0, 0) - at(0, 0, -1, 0)) + inv * (vc - at(1, -1, 0, 0))));
    const double second = 2.0 * coef * inv * (m0 * inv * (at(1, 0, 1, 0) - vc) - m1 * inv * (vc - at(1, 0, -1, 0)));
    const double third =
        coef * inv * (m4 * (inv * (at(1, 0, 0, 1) - vc) + inv * (at(2, 0, 0, zt) - at(2, 0, -1, zt))) -
                      m5 * (inv * (vc - at(1, 0, 0, -1)) + inv * (at(2, 0, 0, zt - 1) - at(2, 0, -1, zt - 1))));
    return vc + ((first + second) + third);
  }
  const double wc = at(2, 0, 0, 0);
  const int xt = IN_PLACE ? 0 : 1, yt = IN_PLACE ? 0 : 1;  // the u column / v row of the high edges
  const double first =
      coef * inv * (m2 * (inv * (at(0, xt, 0, 0) - at(0, xt, 0, -1)) + inv * (at(2, 1, 0, 0) - wc)) -
                    m3 * (inv * (at(0, xt - 1, 0, 0) - at(0, xt - 1, 0, -1)) + inv * (wc - at(2, -1, 0, 0))));
  const double second =
      coef * inv * (m4 * (inv * (at(1, 0, yt, 0) - at(1, 0, yt, -1)) + inv * (at(2, 0, 1, 0) - wc)) -
                    m5 * (inv * (at(1, 0, yt - 1, 0) - at(1, 0, yt - 1, -1)) + inv * (wc - at(2, 0, -1, 0))));
  const double third = 2.0 * coef * inv * (m0 * inv * (at(2, 0, 0, 1) - wc) - m1 * inv * (wc - at(2, 0, 0, -1)));
  return wc + ((first + second) + third);
}

// corrected: out = the updated component from the input velocities
template <class T>
__global__ void k_visc_explicit(ExplicitViscosity X, const T* __restrict__ phi, const T* __restrict__ u,
                                const T* __restrict__ v, const T* __restrict__ w, T* __restrict__ out) {
  const Lay& Lf = X.axis == 0 ? X.Lu : (X.axis == 1 ? X.Lv : X.Lw);
  FS_IJK(Lf);
  const int64_t f = Lf.at(i, j, k);
  const int e = X.axis == 0 ? i : (X.axis == 1 ? j : k);
  const int n = X.axis == 0 ? Lf.nx : (X.axis == 1 ? Lf.ny : Lf.nz);
  const T* comp = X.axis == 0 ? u : (X.axis == 1 ? v : w);
  if (e == 0 || e == n - 1) {
    out[f] = comp[f];
    return;
  }
  out[f] = (T)explicit_visc_face<T, false>(X, PhiX<T>{phi, X.Lc}, u, v, w, i, j, k);
}

// in place: the faces of hyperplane i + j + k = s of component X.axis
template <class T>
__global__ void k_visc_explicit_plane(ExplicitViscosity X, const T* __restrict__ phi, T* u, T* v, T* w, int s) {
  const Lay& Lf = X.axis == 0 ? X.Lu : (X.axis == 1 ? X.Lv : X.Lw);
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = s - j - k;
  if (j >= Lf.ny || k >= Lf.nz || i < 0 || i >= Lf.nx) return;
  T* comp = X.axis == 0 ? u : (X.axis == 1 ? v : w);
  comp[Lf.at(i, j, k)] = (T)explicit_visc_face<T, true>(X, PhiX<T>{phi, X.Lc}, u, v, w, i, j, k);
}

template <class T>
int viscosity_explicit(const T* phi, T* u, T* v, T* w, T* ua, T* va, T* wa, const Lay& Lc, const Lay& Lu,
                       const Lay& Lv, const Lay& Lw, double dx, double dt, double rho_neg, double rho_pos,
                       double mu_neg, double mu_pos, int in_place, cudaStream_t s) {
  ExplicitViscosity X{Lc, Lu, Lv, Lw, 0, 1.0 / dx, dt, rho_neg, rho_pos, mu_neg, mu_pos};
  int launches = 0;
  T* outs[3] = {ua, va, wa};
  const Lay* lays[3] = {&Lu, &Lv, &Lw};
  for (int a = 0; a < 3; ++a) {
    X.axis = a;
    const Lay& Lf = *lays[a];
    if (in_place) {
      const dim3 blk(32, 8, 1), grd((Lf.ny + 31) / 32, (Lf.nz + 7) / 8, 1);
      const int planes = Lf.nx + Lf.ny + Lf.nz - 2;
      for (int p = 0; p < planes; ++p) k_visc_explicit_plane<T><<<grd, blk, 0, s>>>(X, phi, u, v, w, p);
      launches += planes;
    } else {
      Launch3 g = launch3(Lf.nx, Lf.ny, Lf.nz);
      k_visc_explicit<T><<<g.grid, g.block, 0, s>>>(X, phi, u, v, w, outs[a]);
      launches += 1;
    }
  }
  return launches;
}

template int viscosity_explicit<float>(const float*, float*, float*, float*, float*, float*, float*, const Lay&,
                                       const Lay&, const Lay&, const Lay&, double, double, double, double, double,
                                       double, int, cudaStream_t);
template int viscosity_explicit<double>(const double*, double*, double*, double*, double*, double*, double*,
                                        const Lay&, const Lay&, const Lay&, const Lay&, double, double, double, double,
                                        double, double, int, cudaStream_t);

template <class T, class V>
void viscosity_system(const T* phi, const T* u, const T* v, const T* w, const Lay& Lc, const Lay& Lu, const Lay& Lv,
                      const Lay& Lw, int axis, double dx, double dt, double rho_neg, double rho_pos, double mu_neg,
                      double mu_pos, V* ax, V* ay, V* az, V* diag, V* rhs, cudaStream_t s) {
  const Lay& Lf = axis == 0 ? Lu : (axis == 1 ? Lv : Lw);
  Launch3 g = launch3(Lf.nx, Lf.ny, Lf.nz);
  if (axis == 0)
    k_visc_system<T, V, 0><<<g.grid, g.block, 0, s>>>(phi, u, v, w, Lc, Lu, Lv, Lw, Lf, 1.0 / dx, dt, rho_neg,
                                                      rho_pos, mu_neg, mu_pos, ax, ay, az, diag, rhs);
  else if (axis == 1)
    k_visc_system<T, V, 1><<<g.grid, g.block, 0, s>>>(phi, u, v, w, Lc, Lu, Lv, Lw, Lf, 1.0 / dx, dt, rho_neg,
                                                      rho_pos, mu_neg, mu_pos, ax, ay, az, diag, rhs);
  else
    k_visc_system<T, V, 2><<<g.grid, g.block, 0, s>>>(phi, u, v, w, Lc, Lu, Lv, Lw, Lf, 1.0 / dx, dt, rho_neg,
                                                      rho_pos, mu_neg, mu_pos, ax, ay, az, diag, rhs);
}

#define FS_VISC_INST(T, V)                                                                                          \
  template void viscosity_system<T, V>(const T*, const T*, const T*, const T*, const Lay&, const Lay&, const Lay&, \
                                       const Lay&, int, double, double, double, double, double, double, V*, V*, V*, \
                                       V*, V*, cudaStream_t);
FS_VISC_INST(float, float)
FS_VISC_INST(double, double)
FS_VISC_INST(float, double)

}  // namespace fsb
