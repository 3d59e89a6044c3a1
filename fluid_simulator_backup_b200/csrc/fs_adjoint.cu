// Adjoint (vector-Jacobian) kernels of the timestep's operators.  The
// primal fields they read (the forward's states, type T) are FP64 or FP32
// (the FP32 context's storage); the bars are FP64 always and every
// derivative is evaluated and accumulated in FP64.
//
// Each kernel takes the bar (adjoint) of an operator's output and adds the
// bars of its inputs.  The discrete operators are differentiated exactly as
// the forward kernels evaluate them; the non-smooth choices (the upwind side
// of WENO5, the Godunov branch of the Sussman step, the sign-preserving
// clamp, the phase of a cell) are frozen at their forward values, which is
// the derivative wherever the forward map is differentiable.
//
//   WENO5 (ADVECTION_METHOD_3D.h:123-183): D = sum_k w_k u_k with
//   w_k = a_k / sum a, a_k = d_k / (eps + IS_k)^2.  Then
//     dD/dr_j = sum_k w_k du_k/dr_j - 2 sum_k w_k (u_k - D) / (eps + IS_k) dIS_k/dr_j,
//   the second term being the derivative through the nonlinear weights.
//   Stencil bars are scattered with FP64 atomics (each sample of a 7-point
//   stencil receives from up to 21 cells); ghost samples of extrapolated
//   fields are folded back into the interior by the transpose of the linear
//   extrapolation, ghost samples of zero-ghost fields are dropped.
#include "fs_kernels.h"

namespace fsb {

namespace {

constexpr double kPi = 3.14159265358979323846;

// ---- WENO5 one side with its gradient w.r.t. the five differences
__device__ __forceinline__ double weno_side_grad(const double r[5], double eps, double g[5]) {
  const double c1312 = 13.0 / 12.0;
  const double t1 = (r[0] - 2.0 * r[1]) + r[2], q1 = (r[0] - 4.0 * r[1]) + 3.0 * r[2];
  const double t2 = (r[1] - 2.0 * r[2]) + r[3], q2 = r[1] - r[3];
  const double t3 = (r[2] - 2.0 * r[3]) + r[4], q3 = (3.0 * r[2] - 4.0 * r[3]) + r[4];
  const double s1 = (c1312 * t1) * t1 + (0.25 * q1) * q1;
  const double s2 = (c1312 * t2) * t2 + (0.25 * q2) * q2;
  const double s3 = (c1312 * t3) * t3 + (0.25 * q3) * q3;
  const double e1 = eps + s1, e2 = eps + s2, e3 = eps + s3;
  const double qq1 = e1 * e1, qq2 = e2 * e2, qq3 = e3 * e3;
  const double b1 = 0.1 * (qq2 * qq3), b2 = 0.6 * (qq1 * qq3), b3 = 0.3 * (qq1 * qq2);
  const double inv = 1.0 / ((b1 + b2) + b3);
  const double w1 = b1 * inv, w2 = b2 * inv, w3 = b3 * inv;
  const double u1 = (r[0] / 3.0 - r[1] * (7.0 / 6.0)) + r[2] * (11.0 / 6.0);
  const double u2 = (r[1] * (-1.0 / 6.0) + r[2] * (5.0 / 6.0)) + r[3] / 3.0;
  const double u3 = (r[2] / 3.0 + r[3] * (5.0 / 6.0)) - r[4] / 6.0;
  const double D = (w1 * u1 + w2 * u2) + w3 * u3;
  // direct part: sum_k w_k du_k/dr
  g[0] = w1 / 3.0;
  g[1] = -w1 * (7.0 / 6.0) - w2 / 6.0;
  g[2] = w1 * (11.0 / 6.0) + w2 * (5.0 / 6.0) + w3 / 3.0;
  g[3] = w2 / 3.0 + w3 * (5.0 / 6.0);
  g[4] = -w3 / 6.0;
  // weights part: -2 w_k (u_k - D)/(eps + IS_k) * dIS_k/dr
  const double k1 = -2.0 * w1 * (u1 - D) / e1, k2 = -2.0 * w2 * (u2 - D) / e2, k3 = -2.0 * w3 * (u3 - D) / e3;
  // dIS1/dr = 13/6 t1 (1,-2,1) + 1/2 q1 (1,-4,3)
  const double a1 = (13.0 / 6.0) * t1, h1 = 0.5 * q1;
  g[0] += k1 * (a1 + h1);
  g[1] += k1 * (-2.0 * a1 - 4.0 * h1);
  g[2] += k1 * (a1 + 3.0 * h1);
  // dIS2/dr = 13/6 t2 (0,1,-2,1) + 1/2 q2 (0,1,0,-1)
  const double a2 = (13.0 / 6.0) * t2, h2 = 0.5 * q2;
  g[1] += k2 * (a2 + h2);
  g[2] += k2 * (-2.0 * a2);
  g[3] += k2 * (a2 - h2);
  // dIS3/dr = 13/6 t3 (0,0,1,-2,1) + 1/2 q3 (0,0,3,-4,1)
  const double a3 = (13.0 / 6.0) * t3, h3 = 0.5 * q3;
  g[2] += k3 * (a3 + 3.0 * h3);
  g[3] += k3 * (-2.0 * a3 - 4.0 * h3);
  g[4] += k3 * (a3 + h3);
  return D;
}

// Bars of the seven samples f[-3..3] (fb[0..6]) of D- (side 0) or D+ (side 1)
// scaled by m.  d_k = inv_h (f[k-3] - f[k-4]), k = 1..6.
__device__ __forceinline__ void weno_pair_bar(const double f[7], double inv_h, double eps, int side, double m,
                                              double fb[7]) {
  double d[7];
  for (int k = 1; k <= 6; ++k) d[k] = inv_h * (f[k] - f[k - 1]);  // samples stored at s + 3
  double r[5], g[5], db[7] = {0, 0, 0, 0, 0, 0, 0};
  if (side == 0) {
    r[0] = d[1]; r[1] = d[2]; r[2] = d[3]; r[3] = d[4]; r[4] = d[5];
    weno_side_grad(r, eps, g);
    for (int q = 0; q < 5; ++q) db[q + 1] = m * g[q];
  } else {
    r[0] = d[6]; r[1] = d[5]; r[2] = d[4]; r[3] = d[3]; r[4] = d[2];
    weno_side_grad(r, eps, g);
    for (int q = 0; q < 5; ++q) db[6 - q] = m * g[q];
  }
  for (int s = 0; s < 7; ++s) fb[s] = 0.0;
  for (int k = 1; k <= 6; ++k) {
    // d_k = inv_h (f[k] - f[k-1]) in 0-based sample storage
    fb[k] += inv_h * db[k];
    fb[k - 1] -= inv_h * db[k];
  }
}

template <class T>
__device__ __forceinline__ void load7(const T* f, int64_t c, int64_t st, double out[7]) {
#pragma unroll
  for (int s = 0; s < 7; ++s) out[s] = f[c + (s - 3) * st];
}

// scatter stencil bars; with `lo`/`n` given, samples whose coordinate along
// the axis falls outside [0, n) are dropped (zero-ghost fields)
__device__ __forceinline__ void scatter7(double* fb_arr, int64_t c, int64_t st, const double fb[7], int e, int n,
                                         bool drop_ghosts) {
#pragma unroll
  for (int s = 0; s < 7; ++s) {
    if (fb[s] == 0.0) continue;
    if (drop_ghosts && (e + s - 3 < 0 || e + s - 3 >= n)) continue;
    atomicAdd(&fb_arr[c + (s - 3) * st], fb[s]);
  }
}

__device__ __forceinline__ double heaviside(double phi, double e) {
  if (phi < -e) return 0.0;
  if (phi > e) return 1.0;
  return 0.5 * ((1.0 + phi / e) + sin(kPi * phi / e) / kPi);
}
__device__ __forceinline__ double heaviside_d(double phi, double e) {
  if (phi < -e || phi > e) return 0.0;
  return 0.5 * (1.0 / e + cos(kPi * phi / e) / e);
}

}  // namespace

// ---------------------------------------------------------------------------
// Level-set WENO5 update: fe = src - dt (uc D_x + vc D_y + wc D_z), out = c1 fe
// (the RK base term is handled by the caller).  fe_bar = c1 * out_bar.
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_adj_weno_levelset(const T* __restrict__ src, const T* __restrict__ u,
                                    const T* __restrict__ v, const T* __restrict__ w,
                                    const double* __restrict__ out_bar, double* src_bar, double* u_bar,
                                    double* v_bar, double* w_bar, Lay L, Lay Lu, Lay Lv, Lay Lw, double inv_h,
                                    double eps, double dt, double c1) {
  FS_IJK(L);
  const int64_t c = L.at(i, j, k);
  const double fb = c1 * out_bar[c];
  if (fb == 0.0) return;
  atomicAdd(&src_bar[c], fb);
  // the forward's cell velocity, summed in the storage type as the forward does
  const double vel[3] = {(double)(u[Lu.at(i + 1, j, k)] + u[Lu.at(i, j, k)]) * 0.5,
                         (double)(v[Lv.at(i, j + 1, k)] + v[Lv.at(i, j, k)]) * 0.5,
                         (double)(w[Lw.at(i, j, k + 1)] + w[Lw.at(i, j, k)]) * 0.5};
  const int64_t st[3] = {1, L.px, L.slab};
  double* vb[3] = {u_bar, v_bar, w_bar};
  const Lay* lv[3] = {&Lu, &Lv, &Lw};
  for (int a = 0; a < 3; ++a) {
    double f[7], sb[7];
    load7(src, c, st[a], f);
    const int side = vel[a] > 0.0 ? 0 : 1;
    // D of the selected side, for the velocity bar
    double d[7];
    for (int q = 1; q <= 6; ++q) d[q] = inv_h * (f[q] - f[q - 1]);
    double r[5], g[5];
    if (side == 0) { r[0] = d[1]; r[1] = d[2]; r[2] = d[3]; r[3] = d[4]; r[4] = d[5]; }
    else { r[0] = d[6]; r[1] = d[5]; r[2] = d[4]; r[3] = d[3]; r[4] = d[2]; }
    const double D = weno_side_grad(r, eps, g);
    const double velb = -dt * D * fb;
    const int ia = a == 0, ja = a == 1, ka = a == 2;
    atomicAdd(&vb[a][lv[a]->at(i + ia, j + ja, k + ka)], 0.5 * velb);
    atomicAdd(&vb[a][lv[a]->at(i, j, k)], 0.5 * velb);
    weno_pair_bar(f, inv_h, eps, side, -dt * vel[a] * fb, sb);
    scatter7(src_bar, c, st[a], sb, 0, 0, false);
  }
}

// Transpose of the ghost extrapolation of k_fill_extrap: every ghost bar is
// distributed over the interior cells its value was extrapolated from, and
// cleared.  ghost(m) = (m+1) f_0 - m f_1 per out-of-range axis (tensor
// product over the axes, as the extrapolation runs x, then y, then z).
__device__ __forceinline__ bool shell_coord_adj(const Lay& L, int64_t t, int& i, int& j, int& k) {
  const int px = L.nx + 2 * GH, py = L.py;
  const int64_t nzs = (int64_t)2 * GH * px * py;
  if (t < nzs) {
    const int64_t s = t / ((int64_t)px * py), r = t % ((int64_t)px * py);
    k = s < GH ? (int)(s - GH) : (int)(L.nz + (s - GH));
    j = (int)(r / px) - GH;
    i = (int)(r % px) - GH;
    return true;
  }
  t -= nzs;
  const int64_t nys = (int64_t)2 * GH * px * L.nz;
  if (t < nys) {
    const int64_t s = t / ((int64_t)px * L.nz), r = t % ((int64_t)px * L.nz);
    j = s < GH ? (int)(s - GH) : (int)(L.ny + (s - GH));
    k = (int)(r / px);
    i = (int)(r % px) - GH;
    return true;
  }
  t -= nys;
  const int64_t nxs = (int64_t)2 * GH * L.ny * L.nz;
  if (t < nxs) {
    const int64_t s = t / ((int64_t)L.ny * L.nz), r = t % ((int64_t)L.ny * L.nz);
    i = s < GH ? (int)(s - GH) : (int)(L.nx + (s - GH));
    k = (int)(r / L.ny);
    j = (int)(r % L.ny);
    return true;
  }
  return false;
}

__device__ __forceinline__ int extrap_terms(int x, int n, int idx[2], double wt[2]) {
  if (x < 0) { idx[0] = 0; idx[1] = 1; wt[0] = 1.0 - x; wt[1] = x; return 2; }        // m = -x: (m+1), -m
  if (x >= n) { const int m = x - n + 1; idx[0] = n - 1; idx[1] = n - 2; wt[0] = m + 1.0; wt[1] = -m; return 2; }
  idx[0] = x; wt[0] = 1.0;
  return 1;
}

__global__ void k_adj_extrap(double* bar, Lay L) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  if (!shell_coord_adj(L, t, i, j, k)) return;
  const int64_t g = L.at(i, j, k);
  const double v = bar[g];
  if (v == 0.0) return;
  bar[g] = 0.0;
  int ix[2], jx[2], kx[2];
  double wi[2], wj[2], wk[2];
  const int ni = extrap_terms(i, L.nx, ix, wi), nj = extrap_terms(j, L.ny, jx, wj), nk = extrap_terms(k, L.nz, kx, wk);
  for (int a = 0; a < ni; ++a)
    for (int b = 0; b < nj; ++b)
      for (int q = 0; q < nk; ++q) atomicAdd(&bar[L.at(ix[a], jx[b], kx[q])], v * wi[a] * wj[b] * wk[q]);
}

// ---------------------------------------------------------------------------
// MAC component WENO5 self-advection: out = comp - dt (uvel D_x + ...)
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_adj_weno_mac(const T* __restrict__ comp, const T* __restrict__ u,
                               const T* __restrict__ v, const T* __restrict__ w,
                               const double* __restrict__ out_bar, double* comp_bar, double* u_bar, double* v_bar,
                               double* w_bar, Lay Lc, Lay Lu, Lay Lv, Lay Lw, int axis, double inv_h, double eps,
                               double dt) {
  FS_IJK(Lc);
  const int64_t c = Lc.at(i, j, k);
  const double ob = out_bar[c];
  if (ob == 0.0) return;
  atomicAdd(&comp_bar[c], ob);
  // the advecting velocity at this face and the faces it averages
  const T* comps[3] = {u, v, w};
  double* bars[3] = {u_bar, v_bar, w_bar};
  const Lay* lays[3] = {&Lu, &Lv, &Lw};
  const int e[3] = {i, j, k};
  const int n[3] = {Lc.nx, Lc.ny, Lc.nz};
  const int64_t st[3] = {1, Lc.px, Lc.slab};
  for (int d = 0; d < 3; ++d) {
    // velocity component d at this face of component `axis`
    int fi[4], fj[4], fk[4], nf;
    if (d == axis) {
      fi[0] = i; fj[0] = j; fk[0] = k; nf = 1;
    } else {
      // faces (i,j,k), (i,j,k)+e_d, and both shifted back along `axis`
      const int di = d == 0, dj = d == 1, dk = d == 2;
      const int ai = axis == 0, aj = axis == 1, ak = axis == 2;
      fi[0] = i; fj[0] = j; fk[0] = k;
      fi[1] = i + di; fj[1] = j + dj; fk[1] = k + dk;
      fi[2] = i - ai; fj[2] = j - aj; fk[2] = k - ak;
      fi[3] = i - ai + di; fj[3] = j - aj + dj; fk[3] = k - ak + dk;
      nf = 4;
    }
    const Lay& Ld = *lays[d];
    double vel;
    if (nf == 1) {
      vel = comps[d][Ld.at(fi[0], fj[0], fk[0])];
    } else {
      // same association as the forward kernel: ((f0 + f1) + f2) + f3
      vel = (((comps[d][Ld.at(fi[0], fj[0], fk[0])] + comps[d][Ld.at(fi[1], fj[1], fk[1])]) +
              comps[d][Ld.at(fi[2], fj[2], fk[2])]) +
             comps[d][Ld.at(fi[3], fj[3], fk[3])]) *
            0.25;
    }
    double f[7], sb[7];
    load7(comp, c, st[d], f);
    const int side = vel > 0.0 ? 0 : 1;
    double dd[7];
    for (int q = 1; q <= 6; ++q) dd[q] = inv_h * (f[q] - f[q - 1]);
    double r[5], g[5];
    if (side == 0) { r[0] = dd[1]; r[1] = dd[2]; r[2] = dd[3]; r[3] = dd[4]; r[4] = dd[5]; }
    else { r[0] = dd[6]; r[1] = dd[5]; r[2] = dd[4]; r[3] = dd[3]; r[4] = dd[2]; }
    const double D = weno_side_grad(r, eps, g);
    const double velb = -dt * D * ob * (nf == 1 ? 1.0 : 0.25);
    for (int q = 0; q < nf; ++q) {
      // faces outside the face grid of component d are zero ghosts
      if (fi[q] < 0 || fj[q] < 0 || fk[q] < 0 || fi[q] >= Ld.nx || fj[q] >= Ld.ny || fk[q] >= Ld.nz) continue;
      atomicAdd(&bars[d][Ld.at(fi[q], fj[q], fk[q])], velb);
    }
    weno_pair_bar(f, inv_h, eps, side, -dt * vel * ob, sb);
    scatter7(comp_bar, c, st[d], sb, e[d], n[d], true);
  }
}

// ---------------------------------------------------------------------------
// Sussman pseudo-step: r = src - dtau s (|grad src|_G - 1), clamped to
// +-eps when it changes sign; out = c1 r (base handled by the caller).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double godunov_sel(double s, double dm, double dp, int& code, bool& shock) {
  const double sm = s * dm, sp = s * dp;
  shock = false;
  if (sp >= 0.0 && sm >= 0.0) { code = 0; return dm; }
  if (sp <= 0.0 && sm <= 0.0) { code = 1; return dp; }
  if (sp > 0.0 && sm < 0.0) { code = 2; return 0.0; }
  shock = true;
  const double ss = s * (fabs(dp) - fabs(dm)) / (dp - dm);
  if (ss > 0.0) { code = 0; return dm; }
  code = 1;
  return dp;
}

template <class T>
__global__ void k_adj_sussman(const T* __restrict__ src, const T* __restrict__ sgn,
                              const double* __restrict__ out_bar, double* src_bar, double* sgn_bar, Lay L,
                              double inv_h, double eps, double dtau, double c1, int typo) {
  FS_IJK(L);
  const int64_t c = L.at(i, j, k);
  const double rb = c1 * out_bar[c];
  if (rb == 0.0) return;
  const int64_t st[3] = {1, L.px, L.slab};
  double f[3][7], dm[3], dp[3];
  for (int a = 0; a < 3; ++a) {
    load7(src, c, st[a], f[a]);
    double d[7], r[5], g[5];
    for (int q = 1; q <= 6; ++q) d[q] = inv_h * (f[a][q] - f[a][q - 1]);
    r[0] = d[1]; r[1] = d[2]; r[2] = d[3]; r[3] = d[4]; r[4] = d[5];
    dm[a] = weno_side_grad(r, eps, g);
    r[0] = d[6]; r[1] = d[5]; r[2] = d[4]; r[3] = d[3]; r[4] = d[2];
    dp[a] = weno_side_grad(r, eps, g);
  }
  const double s = sgn[c];
  int code[3];
  bool sh[3];
  double gsel[3];
  for (int a = 0; a < 3; ++a) gsel[a] = godunov_sel(s, dm[a], dp[a], code[a], sh[a]);
  const bool typo_leaf = typo && sh[0] && sh[1] && code[1] == 1 && code[2] == 2;
  const double G = (gsel[0] * gsel[0] + gsel[1] * gsel[1]) + gsel[2] * gsel[2];
  double mag, gb[3] = {0, 0, 0};
  if (typo_leaf) {
    mag = (sqrt(gsel[0] * gsel[0]) + gsel[1] * gsel[1]) - 1.0;
  } else {
    mag = sqrt(G) - 1.0;
  }
  const double r = src[c] - dtau * s * mag;
  if (s * r < 0.0) return;  // clamped to a constant: no dependence
  atomicAdd(&src_bar[c], rb);
  sgn_bar[c] += -dtau * mag * rb;  // one thread per cell
  const double mb = -dtau * s * rb;
  if (typo_leaf) {
    gb[0] = gsel[0] > 0.0 ? mb : (gsel[0] < 0.0 ? -mb : 0.0);
    gb[1] = 2.0 * gsel[1] * mb;
  } else if (G > 0.0) {
    const double inv = 1.0 / sqrt(G);
    for (int a = 0; a < 3; ++a) gb[a] = mb * gsel[a] * inv;
  }
  for (int a = 0; a < 3; ++a) {
    if (code[a] == 2 || gb[a] == 0.0) continue;
    double sb[7];
    weno_pair_bar(f[a], inv_h, eps, code[a], gb[a], sb);
    scatter7(src_bar, c, st[a], sb, 0, 0, false);
  }
}

// s = p / sqrt(p^2 + dx^2): p_bar += s_bar dx^2 / (p^2 + dx^2)^(3/2)
template <class T>
__global__ void k_adj_sign(const T* __restrict__ phi, const double* __restrict__ sgn_bar, double* phi_bar, Lay L,
                           double dx) {
  FS_IJK(L);
  const int64_t c = L.at(i, j, k);
  const double p = phi[c], q = p * p + dx * dx;
  phi_bar[c] += sgn_bar[c] * dx * dx / (q * sqrt(q));
}

// ---------------------------------------------------------------------------
// Projection.  Forward (corrected mode): b = P0(-div u*/dt), A(phi) p = b,
// val_f = u*_f - dt beta_f (p_c - p_n) / dx on interior faces (beta_f the
// matrix's face coefficient),
// out = c1 val (+ c0 base, handled by the caller).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double inv_rho_of(double phi, double rn, double rp) { return 1.0 / (phi <= 0.0 ? rn : rp); }

// Transpose of the corrected velocity update u_f -= dt inv_h beta_f (p_c - p_n)
// (beta_f the pressure matrix's face coefficient, see k_velocity_correct):
// in_bar = c1 out_bar; p, phi and density bars of the gradient term, beta's
// derivatives as in k_adj_pressure_operator (the phase of each cell frozen).
template <class T>
__global__ void k_adj_velcorr(const double* __restrict__ p, const T* __restrict__ phi,
                              const double* __restrict__ out_bar, double* __restrict__ in_bar, double* p_bar,
                              double* phi_bar, double* rho_bar, Lay Lf, Lay Lc, int axis, double inv_h, double dt,
                              double rn, double rp, double c1) {
  double rbn = 0.0, rbp = 0.0;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i < Lf.nx && j < Lf.ny && k < Lf.nz) {
    const int64_t fc = Lf.at(i, j, k);
    const double vb = c1 * out_bar[fc];
    in_bar[fc] = vb;
    const int e = axis == 0 ? i : (axis == 1 ? j : k);
    const int n = axis == 0 ? Lc.nx : (axis == 1 ? Lc.ny : Lc.nz);
    if (vb != 0.0 && e > 0 && e < n) {
      const int64_t c = Lc.at(i, j, k);
      const int64_t step = axis == 0 ? 1 : (axis == 1 ? Lc.px : Lc.slab);
      const double pc = phi[c], pn = phi[c - step];
      const double vc = inv_rho_of(pc, rn, rp), vn = inv_rho_of(pn, rn, rp);
      const double ac = fabs(pc), an = fabs(pn);
      const double dp = p[c] - p[c - step];
      const bool same = (pc <= 0.0) == (pn <= 0.0);
      const double beta = same ? vc : vc * vn * (an + ac) / (vn * ac + vc * an);
      // val = u* - dt inv_h beta dp
      const double g = -dt * inv_h * beta * vb;  // d val / d p_c
      atomicAdd(&p_bar[c], g);
      atomicAdd(&p_bar[c - step], -g);
      const double gb = -dt * inv_h * dp * vb;   // d val / d beta
      if (same) {
        // beta = v of the common phase, dv/drho = -v^2
        if (pc <= 0.0) rbn += gb * (-vc * vc); else rbp += gb * (-vc * vc);
      } else {
        const double S = an + ac, D = vn * ac + vc * an, D2 = D * D;
        const double dac = vc * vn * an * (vc - vn) / D2, dan = vc * vn * ac * (vn - vc) / D2;
        atomicAdd(&phi_bar[c], gb * dac * (pc > 0.0 ? 1.0 : (pc < 0.0 ? -1.0 : 0.0)));
        atomicAdd(&phi_bar[c - step], gb * dan * (pn > 0.0 ? 1.0 : (pn < 0.0 ? -1.0 : 0.0)));
        const double dvc = vn * vn * S * ac / D2, dvn = vc * vc * S * an / D2;
        const double bvc = gb * dvc * (-vc * vc), bvn = gb * dvn * (-vn * vn);
        if (pc <= 0.0) rbn += bvc; else rbp += bvc;
        if (pn <= 0.0) rbn += bvn; else rbp += bvn;
      }
    }
  }
  rbn = block_sum(rbn);
  __syncthreads();
  rbp = block_sum(rbp);
  if (thread0()) {
    if (rbn != 0.0) atomicAdd(&rho_bar[0], rbn);
    if (rbp != 0.0) atomicAdd(&rho_bar[1], rbp);
  }
}

// u*_bar_f += -(inv_h/dt) (mu_{e-1} - mu_e), mu = lambda - mean(lambda)
// (the transpose of b = P0(-div u*/dt)); sum_lambda is the device sum.
__global__ void k_adj_divergence(const double* __restrict__ lam, const double* __restrict__ sum_lam, double* in_bar,
                                 Lay Lf, Lay Lc, int axis, double inv_h, double inv_dt, double inv_n) {
  FS_IJK(Lf);
  const double mean = sum_lam[0] * inv_n;
  const int e = axis == 0 ? i : (axis == 1 ? j : k);
  const int n = axis == 0 ? Lc.nx : (axis == 1 ? Lc.ny : Lc.nz);
  const int64_t step = axis == 0 ? 1 : (axis == 1 ? Lc.px : Lc.slab);
  double mu_lo = 0.0, mu_hi = 0.0;
  if (e < n) mu_hi = lam[Lc.at(i, j, k)] - mean;
  if (e > 0) mu_lo = lam[Lc.at(i, j, k) - step] - mean;
  in_bar[Lf.at(i, j, k)] += -(inv_h * inv_dt) * (mu_lo - mu_hi);
}

// sum over the interior of a cell field (one value out)
__global__ void k_adj_sum(const double* __restrict__ f, Lay L, double* partials, unsigned int* ticket, double* out) {
  double s = 0.0;
  Cursor cur;
  for (cur.init(L); cur.valid(L); cur.next(L)) s += f[L.at(cur.i, cur.j, cur.k)];
  s = block_sum(s);
  double tot;
  if (grid_reduce_sum(s, partials, ticket, &tot)) out[0] = tot;
}

// phi and density bars of -lambda^T (dA/dtheta) p: per cell, its three low
// faces and (cell 0) the deflation term.  A p = sum_f beta_f inv2 (p_c - p_n)
// per face, beta = vc vn (ac + an) / (vn ac + vc an) with v = 1/rho of the
// cell's phase and a = |phi|.
template <class T>
__global__ void k_adj_pressure_operator(const T* __restrict__ phi, const double* __restrict__ lam,
                                        const double* __restrict__ p, double* phi_bar, double* rho_bar, Lay Lc,
                                        double rn, double rp, double inv2, int deflate) {
  double rbn = 0.0, rbp = 0.0;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i < Lc.nx && j < Lc.ny && k < Lc.nz) {
    const int64_t c = Lc.at(i, j, k);
    const double pc = phi[c], vc = inv_rho_of(pc, rn, rp), ac = fabs(pc);
    const int64_t step[3] = {1, Lc.px, Lc.slab};
    const bool has[3] = {i > 0, j > 0, k > 0};
    for (int a = 0; a < 3; ++a) {
      if (!has[a]) continue;
      const int64_t nb = c - step[a];
      const double pn = phi[nb], vn = inv_rho_of(pn, rn, rp), an = fabs(pn);
      const double gf = -(lam[c] - lam[nb]) * (p[c] - p[nb]) * inv2;  // bar of beta
      if (gf == 0.0) continue;
      if ((pc <= 0.0) == (pn <= 0.0)) {
        // same phase: beta = v
        if (pc <= 0.0) rbn += gf * (-vc * vc); else rbp += gf * (-vc * vc);
        continue;
      }
      const double S = an + ac, D = vn * ac + vc * an, D2 = D * D;
      const double dac = vc * vn * an * (vc - vn) / D2, dan = vc * vn * ac * (vn - vc) / D2;
      atomicAdd(&phi_bar[c], gf * dac * (pc > 0.0 ? 1.0 : (pc < 0.0 ? -1.0 : 0.0)));
      atomicAdd(&phi_bar[nb], gf * dan * (pn > 0.0 ? 1.0 : (pn < 0.0 ? -1.0 : 0.0)));
      const double dvc = vn * vn * S * ac / D2, dvn = vc * vc * S * an / D2;
      // dv/drho = -v^2 for the cell's phase
      const double bvc = gf * dvc * (-vc * vc), bvn = gf * dvn * (-vn * vn);
      if (pc <= 0.0) rbn += bvc; else rbp += bvc;
      if (pn <= 0.0) rbn += bvn; else rbp += bvn;
    }
    if (deflate && i == 0 && j == 0 && k == 0) {
      // deflation: extra0 = inv2 (e_b + e_d) = 2 inv2 vc
      const double g = -lam[c] * p[c] * 2.0 * inv2 * (-vc * vc);
      if (pc <= 0.0) rbn += g; else rbp += g;
    }
  }
  rbn = block_sum(rbn);
  __syncthreads();
  rbp = block_sum(rbp);
  if (thread0()) {
    if (rbn != 0.0) atomicAdd(&rho_bar[0], rbn);
    if (rbp != 0.0) atomicAdd(&rho_bar[1], rbp);
  }
}

// ---------------------------------------------------------------------------
// Viscosity.  Forward per component a (non-wall rows):
//   (M x)_f = rho_f x_f + sum_arms K mu_arm (x_f - x_nb),  K = k dt inv2
//   r_f = rho_f u_f + dt inv2 sum_t (mu_high_t (hi_a - hi_b) - mu_low_t (lo_a - lo_b))
// with x = 0 on wall faces and beyond.  Given lambda = M^-1 x_bar:
//   u_bar[a]_f += rho_f lambda_f, tangential components get the transpose of
//   the explicit terms, and phi/rho bars come from
//   lambda^T (dr/dtheta) - lambda^T (dM/dtheta) x.
// ---------------------------------------------------------------------------
namespace {
template <class T>
struct PhiXD {  // the forward kernel's one-layer extrapolated phi, with its transpose
  const T* phi;
  Lay L;
  __device__ int terms(int x, int n, int idx[2], double wt[2]) const {
    if (x < 0) { idx[0] = 0; idx[1] = 1; wt[0] = 2.0; wt[1] = -1.0; return 2; }
    if (x >= n) { idx[0] = n - 1; idx[1] = n - 2; wt[0] = 2.0; wt[1] = -1.0; return 2; }
    idx[0] = x; wt[0] = 1.0;
    return 1;
  }
  __device__ double at(int i, int j, int k) const {
    int ix[2], jx[2], kx[2];
    double wi[2], wj[2], wk[2];
    const int ni = terms(i, L.nx, ix, wi), nj = terms(j, L.ny, jx, wj), nk = terms(k, L.nz, kx, wk);
    // same evaluation order as the forward PhiX: x first, then y, then z
    double zsum = 0.0;
    for (int q = 0; q < nk; ++q) {
      double ysum = 0.0;
      for (int b = 0; b < nj; ++b) {
        double xsum = 0.0;
        for (int a = 0; a < ni; ++a) {
          const double val = phi[L.at(ix[a], jx[b], kx[q])];
          xsum = a == 0 ? (ni == 2 ? 2.0 * val : val) : xsum - val;
        }
        ysum = b == 0 ? (nj == 2 ? 2.0 * xsum : xsum) : ysum - xsum;
      }
      zsum = q == 0 ? (nk == 2 ? 2.0 * ysum : ysum) : zsum - ysum;
    }
    return zsum;
  }
  __device__ void scatter(double* bar, int i, int j, int k, double g) const {
    if (g == 0.0) return;
    int ix[2], jx[2], kx[2];
    double wi[2], wj[2], wk[2];
    const int ni = terms(i, L.nx, ix, wi), nj = terms(j, L.ny, jx, wj), nk = terms(k, L.nz, kx, wk);
    for (int a = 0; a < ni; ++a)
      for (int b = 0; b < nj; ++b)
        for (int q = 0; q < nk; ++q) atomicAdd(&bar[L.at(ix[a], jx[b], kx[q])], g * wi[a] * wj[b] * wk[q]);
  }
};
}  // namespace

template <class T>
__global__ void k_adj_visc(const T* __restrict__ phi, const T* __restrict__ ug, const T* __restrict__ vg,
                           const T* __restrict__ wg, const T* __restrict__ x, const double* __restrict__ lam,
                           double* u_bar, double* v_bar, double* w_bar, double* phi_bar, double* rho_bar, Lay Lc,
                           Lay Lu, Lay Lv, Lay Lw, Lay Lf, int axis, double inv_h, double dt, double rn, double rp,
                           double mn, double mp) {
  double rbn = 0.0, rbp = 0.0;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int e_ax = axis == 0 ? i : (axis == 1 ? j : k);
  const int n_ax = axis == 0 ? Lf.nx : (axis == 1 ? Lf.ny : Lf.nz);
  if (i < Lf.nx && j < Lf.ny && k < Lf.nz && !(e_ax == 0 || e_ax == n_ax - 1)) {
    const int64_t f = Lf.at(i, j, k);
    const PhiXD<T> P{phi, Lc};
    const double e = 1.5 / inv_h, inv2 = inv_h * inv_h;
    const int ea[3] = {axis == 0, axis == 1, axis == 2};
    const int li = i - ea[0], lj = j - ea[1], lk = k - ea[2];
    const double lamf = lam[f], xf = x[f];
    const T* comp[3] = {ug, vg, wg};
    double* cbar[3] = {u_bar, v_bar, w_bar};
    const Lay lay[3] = {Lu, Lv, Lw};
    // rho_f and its dependence
    const double mrho = 0.5 * (P.at(li, lj, lk) + P.at(i, j, k));
    const double H = heaviside(mrho, e), dH = heaviside_d(mrho, e);
    const double rho_f = rn + (rp - rn) * H;
    // u_bar[a] += rho_f lambda
    atomicAdd(&cbar[axis][f], rho_f * lamf);
    // The rho_f bar is lambda (u_f - x_f), the viscous change of the face
    // velocity.  It is formed as (K x - E)/rho_f (K the viscous part of the
    // matrix, E the explicit transpose terms: rho_f (u - x) = K x - E for the
    // solved system), accumulated over the arms below, rather than as the
    // difference of the stored velocities, which in FP32 storage cancels to
    // a few digits when the viscous change is small.
    double Kx = 0.0, Ex = 0.0;
    // arms
    for (int d = 0; d < 3; ++d) {
      const int di = d == 0, dj = d == 1, dk = d == 2;
      const double kk = d == axis ? 2.0 : 1.0;
      const double K = kk * dt * inv2;
      // the samples each mu averages, and the average
      int lo_i[4], lo_j[4], lo_k[4], hi_i[4], hi_j[4], hi_k[4], ns;
      if (d == axis) {
        ns = 1;
        lo_i[0] = li; lo_j[0] = lj; lo_k[0] = lk;
        hi_i[0] = i; hi_j[0] = j; hi_k[0] = k;
      } else {
        ns = 4;
        lo_i[0] = li - di; lo_j[0] = lj - dj; lo_k[0] = lk - dk;
        lo_i[1] = li; lo_j[1] = lj; lo_k[1] = lk;
        lo_i[2] = i - di; lo_j[2] = j - dj; lo_k[2] = k - dk;
        lo_i[3] = i; lo_j[3] = j; lo_k[3] = k;
        hi_i[0] = li; hi_j[0] = lj; hi_k[0] = lk;
        hi_i[1] = li + di; hi_j[1] = lj + dj; hi_k[1] = lk + dk;
        hi_i[2] = i; hi_j[2] = j; hi_k[2] = k;
        hi_i[3] = i + di; hi_j[3] = j + dj; hi_k[3] = k + dk;
      }
      const double wgt = ns == 1 ? 1.0 : 0.25;
      double mlo, mhi;
      if (ns == 1) {
        mlo = P.at(lo_i[0], lo_j[0], lo_k[0]);
        mhi = P.at(hi_i[0], hi_j[0], hi_k[0]);
      } else {
        mlo = 0.25 * (((P.at(lo_i[0], lo_j[0], lo_k[0]) + P.at(lo_i[1], lo_j[1], lo_k[1])) + P.at(lo_i[2], lo_j[2], lo_k[2])) +
                      P.at(lo_i[3], lo_j[3], lo_k[3]));
        mhi = 0.25 * (((P.at(hi_i[0], hi_j[0], hi_k[0]) + P.at(hi_i[1], hi_j[1], hi_k[1])) + P.at(hi_i[2], hi_j[2], hi_k[2])) +
                      P.at(hi_i[3], hi_j[3], hi_k[3]));
      }
      const double dmu_lo = (mp - mn) * heaviside_d(mlo, e), dmu_hi = (mp - mn) * heaviside_d(mhi, e);
      const double mu_lo_d = mn + (mp - mn) * heaviside(mlo, e), mu_hi_d = mn + (mp - mn) * heaviside(mhi, e);
      double glo = 0.0, ghi = 0.0;  // bars of mu_low[d], mu_high[d]
      // matrix, low arm: neighbour f - e_d (zero if it is a wall face or beyond)
      {
        const int ni = i - di, nj = j - dj, nk = k - dk;
        const int en = d == 0 ? ni : (d == 1 ? nj : nk);
        const bool nb_wall = (d == axis && (en == 0)) || en < 0;
        const double xn = nb_wall ? 0.0 : x[Lf.at(ni, nj, nk)];
        const double ln = nb_wall ? 0.0 : lam[Lf.at(ni, nj, nk)];
        glo -= K * (lamf - ln) * (xf - xn);
        Kx += K * mu_lo_d * (xf - xn);
      }
      // matrix, high arm: only when the neighbour row does not own it (wall or beyond)
      {
        const int ni = i + di, nj = j + dj, nk = k + dk;
        const int en = d == 0 ? ni : (d == 1 ? nj : nk);
        const int nn = d == 0 ? Lf.nx : (d == 1 ? Lf.ny : Lf.nz);
        const bool nb_wall = (d == axis && en == nn - 1) || en >= nn;
        if (nb_wall) ghi -= K * lamf * xf;
        const double xn = nb_wall ? 0.0 : x[Lf.at(ni, nj, nk)];
        Kx += K * mu_hi_d * (xf - xn);
      }
      // right-hand side: explicit transpose terms for tangential d
      if (d != axis) {
        const T* vt = comp[d];
        const Lay& Lt = lay[d];
        const int ti = di, tj = dj, tk = dk;
        const int64_t ia = Lt.at(i + ti, j + tj, k + tk), ib = Lt.at(i + ti - ea[0], j + tj - ea[1], k + tk - ea[2]);
        const int64_t ja = Lt.at(i, j, k), jb = Lt.at(i - ea[0], j - ea[1], k - ea[2]);
        const double hi_d = vt[ia] - vt[ib], lo_d = vt[ja] - vt[jb];
        ghi += lamf * dt * inv2 * hi_d;
        glo -= lamf * dt * inv2 * lo_d;
        Ex += dt * inv2 * (mu_hi_d * hi_d - mu_lo_d * lo_d);
        // transpose to the tangential component (its ghosts are zero constants)
        // mu values of the forward
        const double ch = lamf * dt * inv2 * mu_hi_d, cl = lamf * dt * inv2 * mu_lo_d;
        auto inside = [&](int a, int b, int q) { return a >= 0 && b >= 0 && q >= 0 && a < Lt.nx && b < Lt.ny && q < Lt.nz; };
        if (inside(i + ti, j + tj, k + tk)) atomicAdd(&cbar[d][ia], ch);
        if (inside(i + ti - ea[0], j + tj - ea[1], k + tk - ea[2])) atomicAdd(&cbar[d][ib], -ch);
        if (inside(i, j, k)) atomicAdd(&cbar[d][ja], -cl);
        if (inside(i - ea[0], j - ea[1], k - ea[2])) atomicAdd(&cbar[d][jb], cl);
      }
      // phi bars through the Heaviside of the averaged samples
      const double plo = glo * dmu_lo * wgt, phi_hi = ghi * dmu_hi * wgt;
      for (int q = 0; q < ns; ++q) {
        P.scatter(phi_bar, lo_i[q], lo_j[q], lo_k[q], plo);
        P.scatter(phi_bar, hi_i[q], hi_j[q], hi_k[q], phi_hi);
      }
    }
    // rho_f bar: lambda (u_f - x_f) = lambda (K x - E)_f / rho_f
    const double rfb = lamf * (Kx - Ex) / rho_f;
    rbn += rfb * (1.0 - H);
    rbp += rfb * H;
    const double pb_rho = rfb * (rp - rn) * dH * 0.5;
    P.scatter(phi_bar, li, lj, lk, pb_rho);
    P.scatter(phi_bar, i, j, k, pb_rho);
  }
  rbn = block_sum(rbn);
  __syncthreads();
  rbp = block_sum(rbp);
  if (thread0()) {
    if (rbn != 0.0) atomicAdd(&rho_bar[0], rbn);
    if (rbp != 0.0) atomicAdd(&rho_bar[1], rbp);
  }
}

// wall rows of a face component: zero (used for x_bar before the transposed
// solve, and for the bar of the no-penetration zeroing)
__global__ void k_adj_zero_walls(double* f, Lay L, int axis) {
  FS_IJK(L);
  const int e = axis == 0 ? i : (axis == 1 ? j : k);
  const int n = axis == 0 ? L.nx : (axis == 1 ? L.ny : L.nz);
  if (e == 0 || e == n - 1) f[L.at(i, j, k)] = 0.0;
}

// out += a * x over the interior
__global__ void k_adj_axpy(double* out, const double* x, double a, Lay L) {
  FS_IJK(L);
  const int64_t c = L.at(i, j, k);
  out[c] += a * x[c];
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <class T>
void adj_weno_levelset(const T* src, const T* u, const T* v, const T* w, const double* out_bar, double* src_bar,
                       double* u_bar, double* v_bar, double* w_bar, const Lay& L, const Lay& Lu, const Lay& Lv,
                       const Lay& Lw, double dx, double eps, double dt, double c1, cudaStream_t s) {
  Launch3 g = launch3(L.nx, L.ny, L.nz, 32, 4, 2);
  k_adj_weno_levelset<T><<<g.grid, g.block, 0, s>>>(src, u, v, w, out_bar, src_bar, u_bar, v_bar, w_bar, L, Lu, Lv,
                                                    Lw, 1.0 / dx, eps, dt, c1);
}

void adj_extrap(double* bar, const Lay& L, cudaStream_t s) {
  const int64_t wx = L.nx + 2 * GH;
  const int64_t n = (int64_t)2 * GH * wx * L.py + (int64_t)2 * GH * wx * L.nz + (int64_t)2 * GH * L.ny * L.nz;
  k_adj_extrap<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(bar, L);
}

template <class T>
void adj_weno_mac(const T* comp, const T* u, const T* v, const T* w, const double* out_bar, double* comp_bar,
                  double* u_bar, double* v_bar, double* w_bar, const Lay& Lc, const Lay& Lu, const Lay& Lv,
                  const Lay& Lw, int axis, double dx, double eps, double dt, cudaStream_t s) {
  Launch3 g = launch3(Lc.nx, Lc.ny, Lc.nz, 32, 4, 2);
  k_adj_weno_mac<T><<<g.grid, g.block, 0, s>>>(comp, u, v, w, out_bar, comp_bar, u_bar, v_bar, w_bar, Lc, Lu, Lv, Lw,
                                               axis, 1.0 / dx, eps, dt);
}

template <class T>
void adj_sussman(const T* src, const T* sgn, const double* out_bar, double* src_bar, double* sgn_bar, const Lay& L,
                 double dx, double eps, double dtau, double c1, int typo, cudaStream_t s) {
  Launch3 g = launch3(L.nx, L.ny, L.nz, 32, 4, 2);
  k_adj_sussman<T><<<g.grid, g.block, 0, s>>>(src, sgn, out_bar, src_bar, sgn_bar, L, 1.0 / dx, eps, dtau, c1, typo);
}

template <class T>
void adj_sign(const T* phi, const double* sgn_bar, double* phi_bar, const Lay& L, double dx, cudaStream_t s) {
  Launch3 g = launch3(L.nx, L.ny, L.nz);
  k_adj_sign<T><<<g.grid, g.block, 0, s>>>(phi, sgn_bar, phi_bar, L, dx);
}

template <class T>
void adj_velcorr(const double* p, const T* phi, const double* out_bar, double* in_bar, double* p_bar, double* phi_bar,
                 double* rho_bar, const Lay& Lf, const Lay& Lc, int axis, double dx, double dt, double rn, double rp,
                 double c1, cudaStream_t s) {
  Launch3 g = launch3(Lf.nx, Lf.ny, Lf.nz);
  k_adj_velcorr<T><<<g.grid, g.block, 0, s>>>(p, phi, out_bar, in_bar, p_bar, phi_bar, rho_bar, Lf, Lc, axis,
                                              1.0 / dx, dt, rn, rp, c1);
}

void adj_divergence(const double* lam, const double* sum_lam, double* in_bar, const Lay& Lf, const Lay& Lc, int axis,
                    double dx, double dt, cudaStream_t s) {
  Launch3 g = launch3(Lf.nx, Lf.ny, Lf.nz);
  k_adj_divergence<<<g.grid, g.block, 0, s>>>(lam, sum_lam, in_bar, Lf, Lc, axis, 1.0 / dx, 1.0 / dt,
                                              1.0 / ((double)Lc.nx * Lc.ny * Lc.nz));
}

void adj_sum(const double* f, const Lay& L, double* partials, unsigned int* ticket, double* out, cudaStream_t s) {
  k_adj_sum<<<pcg_blocks(L), kRedThreads, 0, s>>>(f, L, partials, ticket, out);
}

template <class T>
void adj_pressure_operator(const T* phi, const double* lam, const double* p, double* phi_bar, double* rho_bar,
                           const Lay& Lc, double dx, double rn, double rp, int deflate, cudaStream_t s) {
  Launch3 g = launch3(Lc.nx, Lc.ny, Lc.nz);
  k_adj_pressure_operator<T><<<g.grid, g.block, 0, s>>>(phi, lam, p, phi_bar, rho_bar, Lc, rn, rp, 1.0 / (dx * dx),
                                                        deflate);
}

template <class T>
void adj_visc(const T* phi, const T* ug, const T* vg, const T* wg, const T* x, const double* lam, double* u_bar,
              double* v_bar, double* w_bar, double* phi_bar, double* rho_bar, const Lay& Lc, const Lay& Lu,
              const Lay& Lv, const Lay& Lw, int axis, double dx, double dt, double rn, double rp, double mn,
              double mp, cudaStream_t s) {
  const Lay& Lf = axis == 0 ? Lu : (axis == 1 ? Lv : Lw);
  Launch3 g = launch3(Lf.nx, Lf.ny, Lf.nz);
  k_adj_visc<T><<<g.grid, g.block, 0, s>>>(phi, ug, vg, wg, x, lam, u_bar, v_bar, w_bar, phi_bar, rho_bar, Lc, Lu, Lv,
                                           Lw, Lf, axis, 1.0 / dx, dt, rn, rp, mn, mp);
}

void adj_zero_walls(double* f, const Lay& L, int axis, cudaStream_t s) {
  Launch3 g = launch3(L.nx, L.ny, L.nz);
  k_adj_zero_walls<<<g.grid, g.block, 0, s>>>(f, L, axis);
}

void adj_axpy(double* out, const double* x, double a, const Lay& L, cudaStream_t s) {
  Launch3 g = launch3(L.nx, L.ny, L.nz);
  k_adj_axpy<<<g.grid, g.block, 0, s>>>(out, x, a, L);
}

#define FS_ADJ_INST(T)                                                                                            \
  template void adj_weno_levelset<T>(const T*, const T*, const T*, const T*, const double*, double*, double*,      \
                                     double*, double*, const Lay&, const Lay&, const Lay&, const Lay&, double,       \
                                     double, double, double, cudaStream_t);                                          \
  template void adj_weno_mac<T>(const T*, const T*, const T*, const T*, const double*, double*, double*, double*,  \
                                double*, const Lay&, const Lay&, const Lay&, const Lay&, int, double, double, double, \
                                cudaStream_t);                                                                       \
  template void adj_sussman<T>(const T*, const T*, const double*, double*, double*, const Lay&, double, double,     \
                               double, double, int, cudaStream_t);                                                   \
  template void adj_sign<T>(const T*, const double*, double*, const Lay&, double, cudaStream_t);                     \
  template void adj_velcorr<T>(const double*, const T*, const double*, double*, double*, double*, double*,         \
                               const Lay&, const Lay&, int, double, double, double, double, double, cudaStream_t);   \
  template void adj_pressure_operator<T>(const T*, const double*, const double*, double*, double*, const Lay&,      \
                                         double, double, double, int, cudaStream_t);                                      \
  template void adj_visc<T>(const T*, const T*, const T*, const T*, const T*, const double*, double*, double*,      \
                            double*, double*, double*, const Lay&, const Lay&, const Lay&, const Lay&, int, double,  \
                            double, double, double, double, double, cudaStream_t);

FS_ADJ_INST(float)
FS_ADJ_INST(double)

}  // namespace fsb
