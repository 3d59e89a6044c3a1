// Variable-density ghost-fluid pressure projection, matrix free
// (PROJECTION_3D.h:416-1449, POISSON_SOLVER_3D.h:165-252, 1030-1214).
//
//   divergence_rhs   b = -(div u)/dt and sum(b)           (DetermineDivergence, :681-744)
//   subtract_mean    b -= mean(b), ||b||^2                 (POISSON_SOLVER_3D.h:225-246)
//   build_pressure_operator  beta on faces and the diagonal from phi
//                    (POISSON_SOLVER_3D.h:1075-1214; no CSR is ever built)
//   defect_residual  r64 = b - A64 p64 with A64 evaluated on the fly in FP64
//                    from phi: the FP64 residual of the FP32_REFINE path
//   velocity_correct u -= dt grad p / rho (UpdateVelocityByPressureGradient-
//                    VariableDensity, :1099-1449), fused with the RK combine
#include <cuda_bf16.h>

#include "fs_kernels.h"

namespace fsb {

// beta of the face between cells with (1/rho, |phi|) = (vc, ac) and (vn, an),
// written as the reference's right arm: vc*vn*(an+ac)/(vn*ac + vc*an).
__device__ __forceinline__ double face_beta(double vc, double vn, double ac, double an) {
  return vc * vn * (an + ac) / (vn * ac + vc * an);
}

template <class T>
__device__ __forceinline__ double inv_rho(T phi, double rn, double rp) {
  return 1.0 / ((double)phi <= 0.0 ? rn : rp);
}

template <class T>
__global__ void k_divergence_rhs(const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ w, Lay Lc,
                                 Lay Lu, Lay Lv, Lay Lw, double inv_h, double inv_dt, double* __restrict__ b,
                                 double* __restrict__ div_out, double* partials, unsigned int* ticket,
                                 double* scalars) {
  double bv = 0.0;
  Cursor cur;
  for (cur.init(Lc); cur.valid(Lc); cur.next(Lc)) {
    const int i = cur.i, j = cur.j, k = cur.k;
    const double d = (inv_h * ((double)u[Lu.at(i + 1, j, k)] - (double)u[Lu.at(i, j, k)]) +
                      inv_h * ((double)v[Lv.at(i, j + 1, k)] - (double)v[Lv.at(i, j, k)])) +
                     inv_h * ((double)w[Lw.at(i, j, k + 1)] - (double)w[Lw.at(i, j, k)]);
    const double dv = d * inv_dt;
    const int64_t c = Lc.at(i, j, k);
    div_out[c] = dv;
    b[c] = -dv;
    bv += -dv;
  }
  bv = block_sum(bv);
  double tot;
  if (grid_reduce_sum(bv, partials, ticket, &tot)) scalars[0] = tot;
}

__global__ void k_subtract_mean(double* __restrict__ b, Lay Lc, const double* mean_src, double inv_n,
                                double* partials, unsigned int* ticket, double* out, PipeGeom pg) {
  const double m = inv_n * mean_src[0];
  double bb = 0.0;
  Cursor cur;
  for (cur.init(Lc); cur.valid(Lc); cur.next(Lc)) {
    if (pipe_solid(pg, cur.i, cur.k)) continue;  // no unknown: b stays 0
    const int64_t c = Lc.at(cur.i, cur.j, cur.k);
    const double v = b[c] - m;
    b[c] = v;
    bb += v * v;
  }
  bb = block_sum(bb);
  double tot;
  if (grid_reduce_sum(bb, partials, ticket, &tot)) out[0] = tot;
}

// Coefficients on the cell layout: ax[c] couples cell c-e_x and c (zero on
// the walls i = 0 and i = nx, the latter a ghost column), likewise ay, az.
// Entries are beta/dx^2, the diagonal is inv_dx2 * sum(beta over the six
// faces) in the reference's order l, r, b, t, d, u; the first cell adds the
// betas of its bottom and down Neumann ghosts (deflation, :1145-1179), and a
// zero sum becomes one.
template <class T, class V>
__global__ void k_pressure_faces(const T* __restrict__ phi, Lay Lc, double rn, double rp, double inv2,
                                 V* __restrict__ ax, V* __restrict__ ay, V* __restrict__ az, PipeGeom pg) {
  // one thread per cell, writing the couplings on its low faces; the
  // (i = nx, j = ny, k = nz) ghost faces stay zero from allocation
  FS_IJK(Lc);
  const int64_t c = Lc.at(i, j, k);
  const double pc = (double)phi[c], vc = inv_rho(phi[c], rn, rp), acv = fabs(pc);
  double bx = 0.0, by = 0.0, bz = 0.0;
  // pipe: a coupling only between two unknowns (a y neighbour shares the
  // cell's wall distance)
  const bool solid = pipe_solid(pg, i, k);
  if (i > 0 && !solid && !pipe_solid(pg, i - 1, k)) {
    const double pn = (double)phi[c - 1];
    bx = face_beta(inv_rho(phi[c - 1], rn, rp), vc, fabs(pn), acv);
  }
  if (j > 0 && !solid) {
    const double pn = (double)phi[c - Lc.px];
    by = face_beta(inv_rho(phi[c - Lc.px], rn, rp), vc, fabs(pn), acv);
  }
  if (k > 0 && !solid && !pipe_solid(pg, i, k - 1)) {
    const double pn = (double)phi[c - Lc.slab];
    bz = face_beta(inv_rho(phi[c - Lc.slab], rn, rp), vc, fabs(pn), acv);
  }
  ax[c] = (V)(bx * inv2);
  ay[c] = (V)(by * inv2);
  az[c] = (V)(bz * inv2);
}

template <class T, class V>
__global__ void k_pressure_diag(const T* __restrict__ phi, Lay Lc, double rn, double rp, double inv2,
                                V* __restrict__ diag, double* __restrict__ extra0, unsigned short* __restrict__ dinv16,
                                int deflate, PipeGeom pg) {
  FS_IJK(Lc);
  const int64_t c = Lc.at(i, j, k);
  if (pipe_solid(pg, i, k)) {
    // a Neumann cell of the pipe, no unknown: no couplings, diagonal 1
    diag[c] = (V)1.0;
    if (dinv16) dinv16[c] = __bfloat16_as_ushort(__float2bfloat16_rn(1.0f));
    return;
  }
  const double pc = (double)phi[c], vc = inv_rho(phi[c], rn, rp), acv = fabs(pc);
  double s = 0.0;
  if (i > 0 && !pipe_solid(pg, i - 1, k)) s += face_beta(vc, inv_rho(phi[c - 1], rn, rp), acv, fabs((double)phi[c - 1]));
  if (i < Lc.nx - 1 && !pipe_solid(pg, i + 1, k))
    s += face_beta(vc, inv_rho(phi[c + 1], rn, rp), acv, fabs((double)phi[c + 1]));
  if (j > 0) s += face_beta(vc, inv_rho(phi[c - Lc.px], rn, rp), acv, fabs((double)phi[c - Lc.px]));
  if (j < Lc.ny - 1) s += face_beta(vc, inv_rho(phi[c + Lc.px], rn, rp), acv, fabs((double)phi[c + Lc.px]));
  if (k > 0 && !pipe_solid(pg, i, k - 1))
    s += face_beta(vc, inv_rho(phi[c - Lc.slab], rn, rp), acv, fabs((double)phi[c - Lc.slab]));
  if (k < Lc.nz - 1 && !pipe_solid(pg, i, k + 1))
    s += face_beta(vc, inv_rho(phi[c + Lc.slab], rn, rp), acv, fabs((double)phi[c + Lc.slab]));
  if (pg.on) {
    // the pipe's first unknown (row 0): the faithful system adds the beta of
    // its down neighbour, a Neumann cell (its other Neumann arms add 0)
    if (i == pg.fi && j == pg.fj && k == pg.fk) {
      double e = 0.0;
      if (deflate) {
        const double pd = (double)phi[c - Lc.slab];
        e = face_beta(vc, inv_rho(phi[c - Lc.slab], rn, rp), acv, fabs(pd));
        s = s + e;
      }
      if (extra0) *extra0 = inv2 * e;
    }
  } else if (i == 0 && j == 0 && k == 0 && !deflate) {
    if (extra0) *extra0 = 0.0;
  } else if (i == 0 && j == 0 && k == 0) {
    // deflation: the ghost 1/rho is the clamped copy of vc and the ghost phi
    // the linear extrapolation 2 phi0 - phi1 along the axis
    const double gb = fabs(2.0 * pc - (double)phi[c + Lc.px]);
    const double gd = fabs(2.0 * pc - (double)phi[c + Lc.slab]);
    const double e_b = vc * vc * (gb + acv) / (vc * gb + vc * acv), e_d = vc * vc * (gd + acv) / (vc * gd + vc * acv);
    s = (s + e_b) + e_d;
    if (extra0) *extra0 = inv2 * (e_b + e_d);
  }
  if (s == 0.0) s = 1.0;
  diag[c] = (V)(inv2 * s);
  if (dinv16) dinv16[c] = __bfloat16_as_ushort(__float2bfloat16_rn((float)(1.0 / (inv2 * s))));
}

// r64 = b - A p64 with A from phi in FP64 (same formulas as the two kernels
// above); also r32 = (float) r64 and ||r64||^2.
// With x32 != nullptr the residual is that of the candidate pressure
// p64 + x32 (the mixed-precision solve's uncommitted correction).
template <class T>
__global__ void k_defect_residual(const T* __restrict__ phi, const double* __restrict__ p, const float* __restrict__ x32,
                                  const double* __restrict__ b, double* __restrict__ r64, float* __restrict__ r32,
                                  Lay Lc, double rn, double rp, double inv2, double* partials, unsigned int* ticket,
                                  double* rr_out, int deflate, PipeGeom pg) {
  double rr = 0.0;
  Cursor cur;
  for (cur.init(Lc); cur.valid(Lc); cur.next(Lc)) {
    const int i = cur.i, j = cur.j, k = cur.k;
    const int64_t c = Lc.at(i, j, k);
    if (pipe_solid(pg, i, k)) {  // no unknown: residual 0
      if (r64) r64[c] = 0.0;
      if (r32) r32[c] = 0.0f;
      continue;
    }
    const double pc = (double)phi[c];
    const double xc = x32 ? p[c] + (double)x32[c] : p[c];
    const int64_t nb[6] = {c - 1, c + 1, c - Lc.px, c + Lc.px, c - Lc.slab, c + Lc.slab};
    const bool ok[6] = {i > 0 && !pipe_solid(pg, i - 1, k), i < Lc.nx - 1 && !pipe_solid(pg, i + 1, k), j > 0,
                        j < Lc.ny - 1, k > 0 && !pipe_solid(pg, i, k - 1), k < Lc.nz - 1 && !pipe_solid(pg, i, k + 1)};
    // flux form with the same face coefficients as the on-the-fly SpMV
    double flux = 0.0;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      if (!ok[q]) continue;
      const double xn = x32 ? p[nb[q]] + (double)x32[nb[q]] : p[nb[q]];
      flux += face_coef(pc, (double)phi[nb[q]], 1.0 / rn, 1.0 / rp) * (xc - xn);
    }
    if (deflate && pg.on && i == pg.fi && j == pg.fj && k == pg.fk) {
      const double pd = (double)phi[c - Lc.slab];
      flux += face_beta(inv_rho(phi[c], rn, rp), inv_rho(phi[c - Lc.slab], rn, rp), fabs(pc), fabs(pd)) * xc;
    } else if (deflate && !pg.on && i == 0 && j == 0 && k == 0) {
      const double vc = inv_rho(phi[c], rn, rp), acv = fabs(pc);
      const double gb = fabs(2.0 * pc - (double)phi[c + Lc.px]);
      const double gd = fabs(2.0 * pc - (double)phi[c + Lc.slab]);
      flux += (vc * vc * (gb + acv) / (vc * gb + vc * acv) + vc * vc * (gd + acv) / (vc * gd + vc * acv)) * xc;
    }
    const double ax = inv2 * flux;
    const double rv = b[c] - ax;
    if (r64) r64[c] = rv;
    if (r32) r32[c] = (float)rv;
    rr += rv * rv;
  }
  rr = block_sum(rr);
  double tot;
  if (grid_reduce_sum(rr, partials, ticket, &tot)) rr_out[0] = tot;
}

__global__ void k_add_correction(double* __restrict__ p, const float* __restrict__ e, Lay Lc) {
  FS_IJK(Lc);
  const int64_t c = Lc.at(i, j, k);
  p[c] += (double)e[c];
}

__device__ __forceinline__ double heaviside_proj(double phi, double e) {
  // PROJECTION_3D.h:1452-1470
  const double ooe = 1.0 / e, oop = 1.0 / 3.14159265358979323846;
  if (phi < -e) return 0.0;
  if (phi > e) return 1.0;
  return (0.5 + phi * ooe * 0.5) + 0.5 * oop * sin(3.14159265358979323846 * phi * ooe);
}

// Pressure-gradient update of one face component.  Face (i,j,k) of
// component `axis` lies between cell c = (i,j,k) and the cell n one step
// back along the axis; wall faces are left alone.  Then the RK combination
// out = c0*base + c1*f (skipped when c0 == 0).
//
// Corrected (the default): u_f -= dt beta_f (p_c - p_n +- a_f)/dx with the
// pressure matrix's own face coefficient beta_f (POISSON_SOLVER_3D.h:1080-1085,
// the same expression and operand order as k_pressure_faces) and, on faces
// whose cells lie in different phases, the same interface jump a_f that the
// right-hand side carries (+ when c is in the phi <= 0 phase).  The update
// is then the discrete gradient the matrix was built from: the corrected
// velocity's divergence is dt times the solve's residual, so it is
// divergence free to the solve tolerance at the interface too.
//
// Faithful (FS_FLAG_FAITHFUL_PROJECTION, PROJECTION_3D.h:1099-1449): same-side
// faces use the sharp 1/rho of cell c, faces with phi_c phi_n <= 0 the
// smeared density of the face-averaged phi, only w is updated, and the first
// cell's bottom face sees the zero ghost pressure.  This is not consistent
// with the matrix, so the interface keeps a divergence residual there.
template <class T>
__global__ void k_velocity_correct(T* __restrict__ f, const T* __restrict__ base, const double* __restrict__ p,
                                   const T* __restrict__ phi, Lay Lf, Lay Lc, int axis, double inv_h, double dt,
                                   double rn, double rp, int faithful, double c0, double c1,
                                   const double* __restrict__ kappa, double sigma) {
  FS_IJK(Lf);
  const int64_t fc = Lf.at(i, j, k);
  double val = (double)f[fc];
  const int e = axis == 0 ? i : (axis == 1 ? j : k);
  const int n = axis == 0 ? Lc.nx : (axis == 1 ? Lc.ny : Lc.nz);
  const bool interior = e > 0 && e < n;
  const int64_t c = Lc.at(i, j, k);
  const int64_t step = axis == 0 ? 1 : (axis == 1 ? Lc.px : Lc.slab);
  if (!faithful) {
    if (interior) {
      const double phc = (double)phi[c], phn = (double)phi[c - step];
      const double vc = inv_rho(phi[c], rn, rp), vn = inv_rho(phi[c - step], rn, rp);
      const double beta = face_beta(vn, vc, fabs(phn), fabs(phc));
      double dp = p[c] - p[c - step];
      if (kappa && (phc <= 0.0) != (phn <= 0.0)) {
        const double jcc = sigma * kappa[c], jcn = sigma * kappa[c - step];
        const double jump = (jcc * fabs(phn) + jcn * fabs(phc)) / (fabs(phn) + fabs(phc));
        dp = phc <= 0.0 ? dp + jump : dp - jump;
      }
      val -= dt * dp * beta * inv_h;
    }
  } else if (axis == 2 && (interior || (i == 0 && j == 0 && k == 0))) {
    const double phc = (double)phi[c];
    // across the bottom wall the ghost phi is the linear extrapolation and
    // the ghost pressure is zero
    const double phn = interior ? (double)phi[c - step] : 2.0 * phc - (double)phi[c + step];
    const double pn = interior ? p[c - step] : 0.0;
    const double dp = p[c] - pn;
    double upd;
    if (phc * phn > 0.0) {
      upd = dt * dp * (1.0 / (phc <= 0.0 ? rn : rp)) * inv_h;
    } else {
      const double ef = 1.5 / inv_h;
      const double rho_f = rn + (rp - rn) * heaviside_proj(0.5 * (phc + phn), ef);
      double jump = 0.0;
      if (kappa) {
        // jc interpolated to the interface (PROJECTION_3D.h:1181); the ghost jc is 0
        const double jcc = sigma * kappa[c], jcn = interior ? sigma * kappa[c - step] : 0.0;
        jump = (jcc * fabs(phn) + jcn * fabs(phc)) / (fabs(phn) + fabs(phc));
      }
      upd = dt * (phc <= 0.0 ? dp + jump : dp - jump) * (1.0 / rho_f) * inv_h;
    }
    val -= upd;
  }
  f[fc] = c0 == 0.0 ? (T)val : (T)(c0 * (double)base[fc] + c1 * val);
}

// ---------------------------------------------------------------------------
// Surface tension (LEVELSET_3D.h:963-1082, POISSON_SOLVER_3D.h:1216-1328)
// ---------------------------------------------------------------------------

// Mean curvature from central differences of phi (ghosts extrapolated):
// kappa = -(px^2 pyy - 2 px py pxy + py^2 pxx + px^2 pzz - 2 px pz pxz
//           + pz^2 pxx + py^2 pzz - 2 py pz pyz + pz^2 pyy) / |grad phi|^3,
// clamped below at -1/dx.  typo reproduces the reference's missing factor 2
// on the py pz pyz term and its dz (not 1/dz) in the zero-gradient
// fallback; where the fallback gradient is zero too (the reference exits
// there) kappa is 0.  kmax: max |kappa| over cells with |phi| < 0.1.
__device__ __forceinline__ double curv_num(double px, double py, double pz, double pxx, double pyy, double pzz,
                                           double pxy, double pxz, double pyz, int typo) {
  double t = px * px * pyy - 2.0 * px * py * pxy;
  t = t + py * py * pxx;
  t = t + px * px * pzz;
  t = t - 2.0 * px * pz * pxz;
  t = t + pz * pz * pxx;
  t = t + py * py * pzz;
  t = t - (typo ? py * pz * pyz : 2.0 * py * pz * pyz);
  return t + pz * pz * pyy;
}

template <class T>
__global__ void k_curvature(const T* __restrict__ phi, double* __restrict__ kappa, Lay L, double dx, int typo,
                            double* kmax) {
  double m = 0.0;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i < L.nx && j < L.ny && k < L.nz) {
    const int64_t c = L.at(i, j, k), sy = L.px, sz = L.slab;
    auto f = [&](int64_t o) { return (double)phi[c + o]; };
    const double inv = 1.0 / dx, o2 = 0.5 / dx, o2sq = 1.0 / (dx * dx);
    const double pc = f(0);
    const double px = (f(1) - f(-1)) * o2, py = (f(sy) - f(-sy)) * o2, pz = (f(sz) - f(-sz)) * o2;
    const double pxx = ((f(1) - 2.0 * pc) + f(-1)) * o2sq;
    const double pyy = ((f(sy) - 2.0 * pc) + f(-sy)) * o2sq;
    const double pzz = ((f(sz) - 2.0 * pc) + f(-sz)) * o2sq;
    const double pxy = ((((f(1 + sy) - f(1 - sy)) - f(-1 + sy)) + f(-1 - sy)) * o2) * o2;
    const double pxz = ((((f(1 + sz) - f(1 - sz)) - f(-1 + sz)) + f(-1 - sz)) * o2) * o2;
    const double pyz = ((((f(sy + sz) - f(sy - sz)) - f(-sy + sz)) + f(-sy - sz)) * o2) * o2;
    const double mag = sqrt((px * px + py * py) + pz * pz);
    const double deno = mag * mag * mag;
    double curv;
    if (deno != 0.0) {
      curv = -curv_num(px, py, pz, pxx, pyy, pzz, pxy, pxz, pyz, typo) * (1.0 / deno);
    } else {
      const double fx = (f(1) - pc) * inv, fy = (f(sy) - pc) * inv, fz = (f(sz) - pc) * (typo ? dx : inv);
      const double fm = sqrt((fx * fx + fy * fy) + fz * fz), fd = fm * fm * fm;
      curv = fd != 0.0 ? -curv_num(fx, fy, fz, pxx, pyy, pzz, pxy, pxz, pyz, typo) * (1.0 / fd) : 0.0;
    }
    const double tol = 1.0 / dx;
    const double kv = curv < -tol ? -tol : curv;
    kappa[c] = kv;
    if (fabs(pc) < 1e-1) m = fabs(kv);
  }
  m = block_max(m);
  if (thread0() && m > 0.0) atomicMax((unsigned long long*)kmax, (unsigned long long)__double_as_longlong(m));
}

// b_c = ((b_c - F_X) - F_Y) - F_Z with the ghost-fluid jump terms of the six
// arms (jc_on_derivative = 0): an arm across the interface carries
// +-inv_dx2 * a * beta, a = (jc_c |phi_n| + jc_n |phi_c|)/(|phi_c| + |phi_n|),
// jc = sigma * kappa, + when the cell is in the phi <= 0 phase.  Only arms
// to interior cells can carry a jump: the reference's system
// (POISSON_SOLVER_3D.h:1216-1328) evaluates the wall arms too, but with the
// ghost phi that ComputeNormals (LEVELSET_3D.h:931) has just filled by
// copying the nearest cell, so a wall arm never crosses the interface; the
// corrected projection has no face to correct there either.  The last block
// stores sum(b) in sum_out for the mean removal.
template <class T>
__global__ void k_jump_rhs(const T* __restrict__ phi, const double* __restrict__ kappa, double sigma,
                           double* __restrict__ b, Lay Lc, double rn, double rp, double inv2, int walls,
                           double* partials, unsigned int* ticket, double* sum_out, PipeGeom pg) {
  double bs = 0.0;
  Cursor cur;
  for (cur.init(Lc); cur.valid(Lc); cur.next(Lc)) {
    const int i = cur.i, j = cur.j, k = cur.k;
    if (pipe_solid(pg, i, k)) continue;  // no unknown: b stays 0
    const int64_t c = Lc.at(i, j, k);
    const double pc = (double)phi[c], ac = fabs(pc);
    const double vc = 1.0 / (pc <= 0.0 ? rn : rp);
    const double jcc = sigma * kappa[c];
    const int64_t step[3] = {1, Lc.px, Lc.slab};
    const int e[3] = {i, j, k};
    const int n[3] = {Lc.nx, Lc.ny, Lc.nz};
    double bv = b[c];
    for (int a = 0; a < 3; ++a) {
      double F = 0.0;
      for (int side = 0; side < 2; ++side) {
        const int64_t nb = side == 0 ? c - step[a] : c + step[a];
        const bool ghost = side == 0 ? e[a] == 0 : e[a] == n[a] - 1;
        if (ghost) continue;
        const double pn = (double)phi[nb], an = fabs(pn);
        const double vn = 1.0 / (pn <= 0.0 ? rn : rp);
        const double jn = sigma * kappa[nb];
        double f = 0.0;
        if ((pc <= 0.0) != (pn <= 0.0)) {
          const double av = (jcc * an + jn * ac) / (ac + an);
          const double beta = side == 0 ? vc * vn * (an + ac) / (vc * an + vn * ac)
                                        : vc * vn * (an + ac) / (vn * ac + vc * an);
          f = pc <= 0.0 ? inv2 * av * beta : -inv2 * av * beta;
        }
        F = side == 0 ? f : F + f;
      }
      bv = bv - F;
    }
    b[c] = bv;
    bs += bv;
  }
  bs = block_sum(bs);
  double tot;
  if (grid_reduce_sum(bs, partials, ticket, &tot)) sum_out[0] = tot;
}

template <class T>
__global__ void k_divergence_norms(const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ w, Lay Lc,
                                   Lay Lu, Lay Lv, Lay Lw, double inv_h, double* partials, unsigned int* ticket,
                                   double* out2) {
  double d2 = 0.0, dm = 0.0;
  Cursor cur;
  for (cur.init(Lc); cur.valid(Lc); cur.next(Lc)) {
    const int i = cur.i, j = cur.j, k = cur.k;
    const double d = (inv_h * ((double)u[Lu.at(i + 1, j, k)] - (double)u[Lu.at(i, j, k)]) +
                      inv_h * ((double)v[Lv.at(i, j + 1, k)] - (double)v[Lv.at(i, j, k)])) +
                     inv_h * ((double)w[Lw.at(i, j, k + 1)] - (double)w[Lw.at(i, j, k)]);
    d2 += d * d;
    dm = fmax(dm, fabs(d));
  }
  const double bm = block_max(dm);
  __syncthreads();
  if (thread0()) atomicMax((unsigned long long*)&out2[1], (unsigned long long)__double_as_longlong(bm));
  d2 = block_sum(d2);
  double tot;
  if (grid_reduce_sum(d2, partials, ticket, &tot)) out2[0] = tot;
}

template <class T>
__global__ void k_absmax(const T* __restrict__ f, Lay L, double* out) {
  double m = 0.0;
  Cursor cur;
  for (cur.init(L); cur.valid(L); cur.next(L)) m = fmax(m, fabs((double)f[L.at(cur.i, cur.j, cur.k)]));
  m = block_max(m);
  if (thread0()) atomicMax((unsigned long long*)out, (unsigned long long)__double_as_longlong(m));
}

template <class S, class D>
__global__ void k_convert(D* __restrict__ dst, const S* __restrict__ src, Lay L) {
  FS_IJK(L);
  const int64_t c = L.at(i, j, k);
  dst[c] = (D)src[c];
}

// packed (x fastest, no ghosts) FP64 <-> padded storage
template <class T>
__global__ void k_pack(double* __restrict__ dst, const T* __restrict__ src, Lay L) {
  FS_IJK(L);
  dst[((int64_t)k * L.ny + j) * L.nx + i] = (double)src[L.at(i, j, k)];
}

template <class T>
__global__ void k_unpack(T* __restrict__ dst, const double* __restrict__ src, Lay L) {
  FS_IJK(L);
  dst[L.at(i, j, k)] = (T)src[((int64_t)k * L.ny + j) * L.nx + i];
}

// ---------------------------------------------------------------------------

template <class T>
void divergence_rhs(const T* u, const T* v, const T* w, const Lay& Lc, const Lay& Lu, const Lay& Lv, const Lay& Lw,
                    double dx, double dt, double* b, double* div_out, double* partials, unsigned int* ticket,
                    double* scalars, cudaStream_t s) {
  k_divergence_rhs<T><<<pcg_blocks(Lc), kRedThreads, 0, s>>>(u, v, w, Lc, Lu, Lv, Lw, 1.0 / dx, 1.0 / dt, b, div_out, partials,
                                                  ticket, scalars);
}

void subtract_mean(double* b, const Lay& Lc, const double* scalars, double* partials, unsigned int* ticket,
                   double* scalars_out, cudaStream_t s, const PipeGeom* pipe) {
  const PipeGeom pg = pipe ? *pipe : PipeGeom{};
  const double inv_n = 1.0 / (pg.on ? (double)pg.cells : (double)Lc.nx * Lc.ny * Lc.nz);
  k_subtract_mean<<<pcg_blocks(Lc), kRedThreads, 0, s>>>(b, Lc, scalars, inv_n, partials, ticket, scalars_out, pg);
}

template <class T, class V>
void build_pressure_operator(const T* phi, const Lay& Lc, double dx, double rho_neg, double rho_pos, V* ax, V* ay, V* az,
                             V* diag, double* extra0, int deflate, cudaStream_t s, unsigned short* dinv16,
                             const PipeGeom* pipe) {
  Launch3 g = launch3(Lc.nx, Lc.ny, Lc.nz);
  const double inv2 = 1.0 / (dx * dx);
  const PipeGeom pg = pipe ? *pipe : PipeGeom{};
  k_pressure_faces<T, V><<<g.grid, g.block, 0, s>>>(phi, Lc, rho_neg, rho_pos, inv2, ax, ay, az, pg);
  k_pressure_diag<T, V><<<g.grid, g.block, 0, s>>>(phi, Lc, rho_neg, rho_pos, inv2, diag, extra0, dinv16, deflate,
                                                    pg);
}

template <class T>
void defect_residual(const T* phi, const double* p64, const float* x32, const double* b, double* r64, float* r32,
                     const Lay& Lc, double dx, double rho_neg, double rho_pos, double* partials, unsigned int* ticket,
                     double* rr_out, int deflate, cudaStream_t s, const PipeGeom* pipe) {
  const PipeGeom pg = pipe ? *pipe : PipeGeom{};
  k_defect_residual<T><<<pcg_blocks(Lc), kRedThreads, 0, s>>>(phi, p64, x32, b, r64, r32, Lc, rho_neg, rho_pos,
                                                              1.0 / (dx * dx), partials, ticket, rr_out, deflate, pg);
}

void add_correction(double* p64, const float* e, const Lay& Lc, cudaStream_t s) {
  Launch3 g = launch3(Lc.nx, Lc.ny, Lc.nz);
  k_add_correction<<<g.grid, g.block, 0, s>>>(p64, e, Lc);
}

template <class T>
void velocity_correct(T* f, const T* base, const double* p, const T* phi, const Lay& Lf, const Lay& Lc, int axis,
                      double dx, double dt, double rho_neg, double rho_pos, int faithful, double c0, double c1,
                      const double* kappa, double sigma, cudaStream_t s) {
  Launch3 g = launch3(Lf.nx, Lf.ny, Lf.nz);
  k_velocity_correct<T><<<g.grid, g.block, 0, s>>>(f, base, p, phi, Lf, Lc, axis, 1.0 / dx, dt, rho_neg, rho_pos,
                                                    faithful, c0, c1, kappa, sigma);
}

template <class T>
void curvature(const T* phi, double* kappa, const Lay& L, double dx, int typo, double* kmax, cudaStream_t s) {
  cudaMemsetAsync(kmax, 0, sizeof(double), s);
  Launch3 g = launch3(L.nx, L.ny, L.nz);
  k_curvature<T><<<g.grid, g.block, 0, s>>>(phi, kappa, L, dx, typo, kmax);
}

template <class T>
void jump_rhs(const T* phi, const double* kappa, double sigma, double* b, const Lay& Lc, double dx, double rho_neg,
              double rho_pos, int walls, double* partials, unsigned int* ticket, double* sum_out, cudaStream_t s,
              const PipeGeom* pipe) {
  const PipeGeom pg = pipe ? *pipe : PipeGeom{};
  k_jump_rhs<T><<<pcg_blocks(Lc), kRedThreads, 0, s>>>(phi, kappa, sigma, b, Lc, rho_neg, rho_pos, 1.0 / (dx * dx),
                                                       walls, partials, ticket, sum_out, pg);
}

template <class T>
void divergence_norms(const T* u, const T* v, const T* w, const Lay& Lc, const Lay& Lu, const Lay& Lv, const Lay& Lw,
                      double dx, double* partials, unsigned int* ticket, double* out2, cudaStream_t s) {
  cudaMemsetAsync(out2 + 1, 0, sizeof(double), s);
  k_divergence_norms<T><<<pcg_blocks(Lc), kRedThreads, 0, s>>>(u, v, w, Lc, Lu, Lv, Lw, 1.0 / dx, partials, ticket, out2);
}

template <class T>
void absmax3(const T* u, const T* v, const T* w, const Lay& Lu, const Lay& Lv, const Lay& Lw, double* out3,
             cudaStream_t s) {
  cudaMemsetAsync(out3, 0, 3 * sizeof(double), s);
  k_absmax<T><<<pcg_blocks(Lu), kRedThreads, 0, s>>>(u, Lu, out3);
  k_absmax<T><<<pcg_blocks(Lv), kRedThreads, 0, s>>>(v, Lv, out3 + 1);
  k_absmax<T><<<pcg_blocks(Lw), kRedThreads, 0, s>>>(w, Lw, out3 + 2);
}

template <class S, class D>
void convert_copy(D* dst, const S* src, const Lay& L, cudaStream_t s) {
  Launch3 g = launch3(L.nx, L.ny, L.nz);
  k_convert<S, D><<<g.grid, g.block, 0, s>>>(dst, src, L);
}

template <class T>
void pack_to_double(double* dst, const T* src, const Lay& L, cudaStream_t s) {
  Launch3 g = launch3(L.nx, L.ny, L.nz);
  k_pack<T><<<g.grid, g.block, 0, s>>>(dst, src, L);
}

template <class T>
void unpack_from_double(T* dst, const double* src, const Lay& L, cudaStream_t s) {
  Launch3 g = launch3(L.nx, L.ny, L.nz);
  k_unpack<T><<<g.grid, g.block, 0, s>>>(dst, src, L);
}

#define FS_PINST(T)                                                                                                  \
  template void divergence_rhs<T>(const T*, const T*, const T*, const Lay&, const Lay&, const Lay&, const Lay&,     \
                                  double, double, double*, double*, double*, unsigned int*, double*, cudaStream_t); \
  template void defect_residual<T>(const T*, const double*, const float*, const double*, double*, float*,         \
                                   const Lay&, double, double, double, double*, unsigned int*, double*, int,        \
                                   cudaStream_t, const PipeGeom*);                                                  \
  template void velocity_correct<T>(T*, const T*, const double*, const T*, const Lay&, const Lay&, int, double,     \
                                    double, double, double, int, double, double, const double*, double,            \
                                    cudaStream_t);                                                                  \
  template void curvature<T>(const T*, double*, const Lay&, double, int, double*, cudaStream_t);                   \
  template void jump_rhs<T>(const T*, const double*, double, double*, const Lay&, double, double, double, int,    \
                            double*, unsigned int*, double*, cudaStream_t, const PipeGeom*);                 \
  template void divergence_norms<T>(const T*, const T*, const T*, const Lay&, const Lay&, const Lay&, const Lay&,   \
                                    double, double*, unsigned int*, double*, cudaStream_t);                         \
  template void absmax3<T>(const T*, const T*, const T*, const Lay&, const Lay&, const Lay&, double*, cudaStream_t); \
  template void pack_to_double<T>(double*, const T*, const Lay&, cudaStream_t);                                     \
  template void unpack_from_double<T>(T*, const double*, const Lay&, cudaStream_t);

FS_PINST(float)
FS_PINST(double)

#define FS_BINST(T, V)                                                                                        \
  template void build_pressure_operator<T, V>(const T*, const Lay&, double, double, double, V*, V*, V*, V*, double*, \
                                              int, cudaStream_t, unsigned short*, const PipeGeom*);
FS_BINST(float, float)
FS_BINST(double, double)
FS_BINST(double, float)
FS_BINST(float, double)
template void convert_copy<float, double>(double*, const float*, const Lay&, cudaStream_t);
template void convert_copy<double, float>(float*, const double*, const Lay&, cudaStream_t);
template void convert_copy<double, double>(double*, const double*, const Lay&, cudaStream_t);
template void convert_copy<float, float>(float*, const float*, const Lay&, cudaStream_t);

}  // namespace fsb
