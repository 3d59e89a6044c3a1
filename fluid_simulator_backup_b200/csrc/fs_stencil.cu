// Level-set and velocity stencil kernels: ghost fills, WENO5 advection
// (ADVECTION_METHOD_3D.h:42-279), Sussman reinitialisation
// (ADVECTION_METHOD_3D.h:745-1637) and the RK stage combiners
// (EULERIAN_FLUID_SOLVER_3D.h:886-1109), templated on the storage/arithmetic
// type (double for the FP64 path, float for FP32_REFINE).
//
// Staging.  The four seven-point stencil kernels (WENO5 level set, WENO5 and
// ENO3 MAC components, Sussman) run on 32 x 8 column tiles that march up a
// chunk of z planes: the stencil field is staged in shared memory as a ring of
// seven (32+6) x (8+6) planes (the tile and its three-cell halo), one new
// plane loaded per output plane with row-contiguous (coalesced) loads, and
// every x, y and z sample of the stencil is read from that ring.  HBM then
// carries each field element about once per kernel instead of up to 19
// times through L1/L2.  The ghost ring of the padded layout supplies the halo
// at the box boundary.
//
// These kernels are FP32/FP64-issue bound rather than HBM bound (about 440
// flops per cell per WENO5 update), so the WENO weights are evaluated with one
// division per side: w_k = d_k prod_{j!=k} q_j / sum_m d_m prod_{j!=m} q_j
// with q = (eps + IS)^2, algebraically equal to the reference's
// (d_k/q_k)/sum(d_m/q_m).  The substencil constants 1/3, 7/6, ... are applied
// as multiplications.  Both change results only at the level of rounding.
#include <algorithm>

#include "fs_kernels.h"

namespace fsb {

// ---------------------------------------------------------------------------
// ghost fills
// ---------------------------------------------------------------------------

// m-th ghost layer (m = 1..3) of the outward linear extrapolation
// ghost(-m) = 2 ghost(-m+1) - ghost(-m+2), evaluated recursively from the
// two boundary values f0 (on the wall) and f1 (one inside) as the reference
// does (FIELD_STRUCTURE_3D.h:1776-1895).
template <class T>
__device__ __forceinline__ T extrap_layer(T f0, T f1, int m) {
  T a = f1, b = f0;  // (layer m-2, layer m-1)
  for (int q = 0; q < m; ++q) {
    T c = T(2) * b - a;
    a = b;
    b = c;
  }
  return b;
}

template <class T>
struct ExtrapField {
  const T* f;
  Lay L;
  // value at (i, j, k) with i, j, k possibly in the ghost ring: extend x
  // first, then y, then z (dimension by dimension).
  __device__ T x_ext(int i, int j, int k) const {
    if (i < 0) return extrap_layer(f[L.at(0, j, k)], f[L.at(1, j, k)], -i);
    if (i >= L.nx) return extrap_layer(f[L.at(L.nx - 1, j, k)], f[L.at(L.nx - 2, j, k)], i - L.nx + 1);
    return f[L.at(i, j, k)];
  }
  __device__ T y_ext(int i, int j, int k) const {
    if (j < 0) return extrap_layer(x_ext(i, 0, k), x_ext(i, 1, k), -j);
    if (j >= L.ny) return extrap_layer(x_ext(i, L.ny - 1, k), x_ext(i, L.ny - 2, k), j - L.ny + 1);
    return x_ext(i, j, k);
  }
  __device__ T z_ext(int i, int j, int k) const {
    if (k < 0) return extrap_layer(y_ext(i, j, 0), y_ext(i, j, 1), -k);
    if (k >= L.nz) return extrap_layer(y_ext(i, j, L.nz - 1), y_ext(i, j, L.nz - 2), k - L.nz + 1);
    return y_ext(i, j, k);
  }
};

// Decode a flat index over the ghost shell: the z slabs (full padded x, y),
// then the y slabs (interior z, full padded x), then the x slabs (interior
// y, z).  Returns false past the end.
__device__ __forceinline__ bool shell_coord(const Lay& L, int64_t t, int& i, int& j, int& k) {
  const int px = L.nx + 2 * GH, py = L.py;  // logical extents: the alignment columns are not part of the shell
  const int64_t nzs = (int64_t)2 * GH * px * py;
  if (t < nzs) {
    const int64_t s = t / ((int64_t)px * py);
    const int64_t r = t % ((int64_t)px * py);
    k = s < GH ? (int)(s - GH) : (int)(L.nz + (s - GH));
    j = (int)(r / px) - GH;
    i = (int)(r % px) - GH;
    return true;
  }
  t -= nzs;
  const int64_t nys = (int64_t)2 * GH * px * L.nz;
  if (t < nys) {
    const int64_t s = t / ((int64_t)px * L.nz);
    const int64_t r = t % ((int64_t)px * L.nz);
    j = s < GH ? (int)(s - GH) : (int)(L.ny + (s - GH));
    k = (int)(r / px);
    i = (int)(r % px) - GH;
    return true;
  }
  t -= nys;
  const int64_t nxs = (int64_t)2 * GH * L.ny * L.nz;
  if (t < nxs) {
    const int64_t s = t / ((int64_t)L.ny * L.nz);
    const int64_t r = t % ((int64_t)L.ny * L.nz);
    i = s < GH ? (int)(s - GH) : (int)(L.nx + (s - GH));
    k = (int)(r / L.ny);
    j = (int)(r % L.ny);
    return true;
  }
  return false;
}

inline int64_t shell_count(const Lay& L) {
  const int64_t wx = L.nx + 2 * GH;
  return (int64_t)2 * GH * wx * L.py + (int64_t)2 * GH * wx * L.nz + (int64_t)2 * GH * L.ny * L.nz;
}

template <class T>
__global__ void k_fill_extrap(T* f, Lay L) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  if (!shell_coord(L, t, i, j, k)) return;
  ExtrapField<T> e{f, L};
  f[L.at(i, j, k)] = e.z_ext(i, j, k);
}

template <class T>
void fill_extrap(T* f, const Lay& L, cudaStream_t s) {
  const int64_t n = shell_count(L);
  k_fill_extrap<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(f, L);
}

// ---------------------------------------------------------------------------
// WENO5
// ---------------------------------------------------------------------------

template <class T>
__device__ __forceinline__ T weno_side(T r1, T r2, T r3, T r4, T r5, T eps) {
  const T c1312 = T(13.0 / 12.0);
  T t = (r1 - T(2) * r2) + r3, q = (r1 - T(4) * r2) + T(3) * r3;
  const T s1 = (c1312 * t) * t + (T(0.25) * q) * q;
  t = (r2 - T(2) * r3) + r4; q = r2 - r4;
  const T s2 = (c1312 * t) * t + (T(0.25) * q) * q;
  t = (r3 - T(2) * r4) + r5; q = (T(3) * r3 - T(4) * r4) + r5;
  const T s3 = (c1312 * t) * t + (T(0.25) * q) * q;
  const T e1 = eps + s1, e2 = eps + s2, e3 = eps + s3;
  const T q1 = e1 * e1, q2 = e2 * e2, q3 = e3 * e3;
  const T b1 = T(0.1) * (q2 * q3), b2 = T(0.6) * (q1 * q3), b3 = T(0.3) * (q1 * q2);
  const T inv = T(1) / ((b1 + b2) + b3);
  const T third = T(1.0 / 3.0), sixth = T(1.0 / 6.0);
  const T u1 = (r1 * third - r2 * T(7.0 / 6.0)) + r3 * T(11.0 / 6.0);
  const T u2 = (r2 * (-sixth) + r3 * T(5.0 / 6.0)) + r4 * third;
  const T u3 = (r3 * third + r4 * T(5.0 / 6.0)) - r5 * sixth;
  return ((b1 * u1 + b2 * u2) + b3 * u3) * inv;
}

// D- and D+ from the 7 samples v[0..6] = f[-3..3] along one axis.
template <class T>
__device__ __forceinline__ void weno_pair7(const T v[7], T inv_h, T eps, T& dm, T& dp) {
  const T d1 = inv_h * (v[1] - v[0]), d2 = inv_h * (v[2] - v[1]), d3 = inv_h * (v[3] - v[2]),
          d4 = inv_h * (v[4] - v[3]), d5 = inv_h * (v[5] - v[4]), d6 = inv_h * (v[6] - v[5]);
  dm = weno_side(d1, d2, d3, d4, d5, eps);
  dp = weno_side(d6, d5, d4, d3, d2, eps);
}

// ---------------------------------------------------------------------------
// shared-memory plane ring of the staged stencil kernels
// ---------------------------------------------------------------------------
constexpr int kTX = 32, kTY = 8;                     // tile (threads) in x and y
constexpr int kRW = kTX + 2 * GH, kRH = kTY + 2 * GH;  // staged plane: tile + halo
constexpr int kRing = 2 * GH + 1;                    // planes k-3 .. k+3

__device__ __forceinline__ int ring_slot(int k) { return ((k % kRing) + kRing) % kRing; }

// Plane k of f (halo included) into its ring slot: row-contiguous loads of
// the (32+6) x (8+6) window; halo cells beyond the ghost ring (i >= nx+3 or
// j >= ny+3, only at the tile past the box edge) are not needed and skipped.
template <class T>
__device__ __forceinline__ void stage_plane(T* ring, const T* __restrict__ f, const Lay& L, int i0, int j0, int k) {
  T* dst = ring + ring_slot(k) * (kRW * kRH);
  const int tid = threadIdx.x + kTX * threadIdx.y;
  for (int t = tid; t < kRW * kRH; t += kTX * kTY) {
    const int x = t % kRW, y = t / kRW;
    const int gi = i0 - GH + x, gj = j0 - GH + y;
    if (gi < L.nx + GH && gj < L.ny + GH) dst[t] = f[L.at(gi, gj, k)];
  }
}

// The seven samples of (tx, ty) in plane k along x, y and z from the ring.
template <class T>
__device__ __forceinline__ void ring_samples(const T* ring, int k, T vx[7], T vy[7], T vz[7]) {
  const int tx = threadIdx.x + GH, ty = threadIdx.y + GH;
  const T* pc = ring + ring_slot(k) * (kRW * kRH);
#pragma unroll
  for (int o = 0; o < 7; ++o) {
    vx[o] = pc[ty * kRW + tx + o - GH];
    vy[o] = pc[(ty + o - GH) * kRW + tx];
    vz[o] = ring[ring_slot(k + o - GH) * (kRW * kRH) + ty * kRW + tx];
  }
}

// Grid of a staged kernel: xy tiles times z chunks, enough blocks to fill
// the GPU a few times over (each chunk re-stages six halo planes).
struct StagedGrid {
  dim3 grid;
  int kchunk;
};
inline StagedGrid staged_grid(const Lay& L) {
  static int sms = 0;
  if (sms <= 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  }
  const int tx = (L.nx + kTX - 1) / kTX, ty = (L.ny + kTY - 1) / kTY;
  const int want = 8 * sms;
  const int chunks = std::max(1, std::min(L.nz, (want + tx * ty - 1) / (tx * ty)));
  const int kchunk = (L.nz + chunks - 1) / chunks;
  StagedGrid g;
  g.grid = dim3(tx, ty, (L.nz + kchunk - 1) / kchunk);
  g.kchunk = kchunk;
  return g;
}

// out = c0*base + c1*(src - dt*(u.grad src)), the level-set update at cell
// centres; u, v, w are the MAC faces (zero ghosts).  With c0 == 0 the
// combination is skipped and out is the forward-Euler value.
template <class T>
__global__ void __launch_bounds__(kTX * kTY) k_weno5_levelset(const T* __restrict__ src, const T* __restrict__ base,
                                                           T* __restrict__ out, const T* __restrict__ u,
                                                           const T* __restrict__ v, const T* __restrict__ w, Lay L,
                                                           Lay Lu, Lay Lv, Lay Lw, T inv_h, T eps, T dt, T c0, T c1,
                                                           int kchunk, PipeGeom pipe) {
  __shared__ T ring[kRing * kRW * kRH];
  const int i0 = blockIdx.x * kTX, j0 = blockIdx.y * kTY;
  const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  const int k0 = blockIdx.z * kchunk, k1 = min(L.nz, k0 + kchunk);
  const bool valid = i < L.nx && j < L.ny;
  for (int kk = k0 - GH; kk < k0 + GH; ++kk) stage_plane(ring, src, L, i0, j0, kk);
  for (int k = k0; k < k1; ++k) {
    stage_plane(ring, src, L, i0, j0, k + GH);
    __syncthreads();
    if (valid) {
      T vx[7], vy[7], vz[7];
      ring_samples(ring, k, vx, vy, vz);
      T dxm, dxp, dym, dyp, dzm, dzp;
      weno_pair7(vx, inv_h, eps, dxm, dxp);
      weno_pair7(vy, inv_h, eps, dym, dyp);
      weno_pair7(vz, inv_h, eps, dzm, dzp);
      const int64_t c = L.at(i, j, k);
      const T uc = (u[Lu.at(i + 1, j, k)] + u[Lu.at(i, j, k)]) * T(0.5);
      const T vc = (v[Lv.at(i, j + 1, k)] + v[Lv.at(i, j, k)]) * T(0.5);
      const T wc = (w[Lw.at(i, j, k + 1)] + w[Lw.at(i, j, k)]) * T(0.5);
      T fe =
          vx[3] - dt * ((uc * (uc > T(0) ? dxm : dxp) + vc * (vc > T(0) ? dym : dyp)) + wc * (wc > T(0) ? dzm : dzp));
      // pipe mode: cells outside the pipe keep their value
      // (ADVECTION_METHOD_3D.h:293-296)
      if (pipe.on && pipe_wall_distance(pipe, 0, i, k) > 0.0) fe = vx[3];
      out[c] = c0 == T(0) ? fe : c0 * base[c] + c1 * fe;
    }
    __syncthreads();
  }
}

// The velocities that advect face (i,j,k) of component `axis`: its own
// component, the four-face averages of the other two.
template <class T>
__device__ __forceinline__ void mac_velocity(const T* __restrict__ u, const T* __restrict__ v,
                                             const T* __restrict__ w, const Lay& Lu, const Lay& Lv, const Lay& Lw,
                                             int axis, int i, int j, int k, T& uvel, T& vvel, T& wvel) {
  if (axis == 0) {
    uvel = u[Lu.at(i, j, k)];
    vvel = (((v[Lv.at(i, j, k)] + v[Lv.at(i, j + 1, k)]) + v[Lv.at(i - 1, j, k)]) + v[Lv.at(i - 1, j + 1, k)]) * T(0.25);
    wvel = (((w[Lw.at(i, j, k)] + w[Lw.at(i, j, k + 1)]) + w[Lw.at(i - 1, j, k)]) + w[Lw.at(i - 1, j, k + 1)]) * T(0.25);
  } else if (axis == 1) {
    uvel = (((u[Lu.at(i, j, k)] + u[Lu.at(i + 1, j, k)]) + u[Lu.at(i, j - 1, k)]) + u[Lu.at(i + 1, j - 1, k)]) * T(0.25);
    vvel = v[Lv.at(i, j, k)];
    wvel = (((w[Lw.at(i, j, k)] + w[Lw.at(i, j, k + 1)]) + w[Lw.at(i, j - 1, k)]) + w[Lw.at(i, j - 1, k + 1)]) * T(0.25);
  } else {
    uvel = (((u[Lu.at(i, j, k)] + u[Lu.at(i + 1, j, k)]) + u[Lu.at(i, j, k - 1)]) + u[Lu.at(i + 1, j, k - 1)]) * T(0.25);
    vvel = (((v[Lv.at(i, j, k)] + v[Lv.at(i, j + 1, k)]) + v[Lv.at(i, j, k - 1)]) + v[Lv.at(i, j + 1, k - 1)]) * T(0.25);
    wvel = w[Lw.at(i, j, k)];
  }
}

// MAC component self-advection on every face of component `axis` (wall
// faces included, as the reference's loop covers the whole face grid).
template <class T>
__global__ void __launch_bounds__(kTX * kTY) k_weno5_mac(const T* __restrict__ comp, T* __restrict__ out,
                                                      const T* __restrict__ u, const T* __restrict__ v,
                                                      const T* __restrict__ w, Lay Lc, Lay Lu, Lay Lv, Lay Lw,
                                                      int axis, T inv_h, T eps, T dt, int kchunk) {
  __shared__ T ring[kRing * kRW * kRH];
  const int i0 = blockIdx.x * kTX, j0 = blockIdx.y * kTY;
  const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  const int k0 = blockIdx.z * kchunk, k1 = min(Lc.nz, k0 + kchunk);
  const bool valid = i < Lc.nx && j < Lc.ny;
  for (int kk = k0 - GH; kk < k0 + GH; ++kk) stage_plane(ring, comp, Lc, i0, j0, kk);
  for (int k = k0; k < k1; ++k) {
    stage_plane(ring, comp, Lc, i0, j0, k + GH);
    __syncthreads();
    if (valid) {
      T uvel, vvel, wvel;
      mac_velocity(u, v, w, Lu, Lv, Lw, axis, i, j, k, uvel, vvel, wvel);
      T vx[7], vy[7], vz[7];
      ring_samples(ring, k, vx, vy, vz);
      T dxm, dxp, dym, dyp, dzm, dzp;
      weno_pair7(vx, inv_h, eps, dxm, dxp);
      weno_pair7(vy, inv_h, eps, dym, dyp);
      weno_pair7(vz, inv_h, eps, dzm, dzp);
      out[Lc.at(i, j, k)] = vx[3] - dt * ((uvel * (uvel > T(0) ? dxm : dxp) + vvel * (vvel > T(0) ? dym : dyp)) +
                                          wvel * (wvel > T(0) ? dzm : dzp));
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// ENO3 (ADVECTION_METHOD_3D.h:1639-1934)
// ---------------------------------------------------------------------------

// D- and D+ along a stride from the 7 samples f[-3..3]: divided differences
// d1 (scaled 1/dx), d2 (1/(2dx)), d3 ((1/dx)/3); each side takes the stencil
// with the smaller |d2|, then the smaller |d3|.
template <class T>
__device__ __forceinline__ void eno3_pair7(const T v[7], T h, T inv, T o2, T o3, T& dm, T& dp) {
  T d1[6], d2[5], d3[4];  // d1[q]: samples q+1 - q (s = q-3); d2[q] from d1[q+1], d1[q]; d3[q] from d2[q+1], d2[q]
#pragma unroll
  for (int q = 0; q < 6; ++q) d1[q] = inv * (v[q + 1] - v[q]);
#pragma unroll
  for (int q = 0; q < 5; ++q) d2[q] = o2 * (d1[q + 1] - d1[q]);
#pragma unroll
  for (int q = 0; q < 4; ++q) d3[q] = o3 * (d2[q + 1] - d2[q]);
  // in the reference's names: d1_n1 = d1[2], d1_0 = d1[3]; d2_n1 = d2[1],
  // d2_0 = d2[2], d2_p1 = d2[3]; d3_n2 = d3[0], d3_n1 = d3[1], d3_0 = d3[2], d3_p1 = d3[3]
  const T two = T(2);
  if (fabs(d2[1]) <= fabs(d2[2])) {
    dm = fabs(d3[0]) <= fabs(d3[1]) ? (d1[2] + d2[1] * h) + two * d3[0] * h * h : (d1[2] + d2[1] * h) + two * d3[1] * h * h;
  } else {
    dm = fabs(d3[1]) <= fabs(d3[2]) ? (d1[2] + d2[2] * h) - d3[1] * h * h : (d1[2] + d2[2] * h) - d3[2] * h * h;
  }
  if (fabs(d2[2]) <= fabs(d2[3])) {
    dp = fabs(d3[1]) <= fabs(d3[2]) ? (d1[3] - d2[2] * h) - d3[1] * h * h : (d1[3] - d2[2] * h) - d3[2] * h * h;
  } else {
    dp = fabs(d3[2]) <= fabs(d3[3]) ? (d1[3] - d2[3] * h) + two * d3[2] * h * h : (d1[3] - d2[3] * h) + two * d3[3] * h * h;
  }
}

// MAC component self-advection with ENO3 (the reference's use_3rd_eno_v,
// ADVECTION_3D.h:323-325), every face of component `axis`.
template <class T>
__global__ void __launch_bounds__(kTX * kTY) k_eno3_mac(const T* __restrict__ comp, T* __restrict__ out,
                                                     const T* __restrict__ u, const T* __restrict__ v,
                                                     const T* __restrict__ w, Lay Lc, Lay Lu, Lay Lv, Lay Lw,
                                                     int axis, T h, T dt, int kchunk) {
  __shared__ T ring[kRing * kRW * kRH];
  const int i0 = blockIdx.x * kTX, j0 = blockIdx.y * kTY;
  const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  const int k0 = blockIdx.z * kchunk, k1 = min(Lc.nz, k0 + kchunk);
  const bool valid = i < Lc.nx && j < Lc.ny;
  const T inv = T(1) / h, o2 = T(0.5) / h, o3 = inv * T(1) / T(3);
  for (int kk = k0 - GH; kk < k0 + GH; ++kk) stage_plane(ring, comp, Lc, i0, j0, kk);
  for (int k = k0; k < k1; ++k) {
    stage_plane(ring, comp, Lc, i0, j0, k + GH);
    __syncthreads();
    if (valid) {
      T uvel, vvel, wvel;
      mac_velocity(u, v, w, Lu, Lv, Lw, axis, i, j, k, uvel, vvel, wvel);
      T vx[7], vy[7], vz[7];
      ring_samples(ring, k, vx, vy, vz);
      T dxm, dxp, dym, dyp, dzm, dzp;
      eno3_pair7(vx, h, inv, o2, o3, dxm, dxp);
      eno3_pair7(vy, h, inv, o2, o3, dym, dyp);
      eno3_pair7(vz, h, inv, o2, o3, dzm, dzp);
      out[Lc.at(i, j, k)] = vx[3] - dt * ((uvel * (uvel > T(0) ? dxm : dxp) + vvel * (vvel > T(0) ? dym : dyp)) +
                                          wvel * (wvel > T(0) ? dzm : dzp));
    }
    __syncthreads();
  }
}

// The vertical pipe's ENO3 self-advection of component `axis`
// (ADVECTION_METHOD_3D.h:1935-2240): faces inside the pipe and off the
// fixed centre line take the ENO3 upwind update in place, the x and z
// derivatives from the guarded copies gx, gz, the y derivative from the
// masked periodic copy gen, the advecting velocities from the masked
// periodic copies ug, vg, wg; the other faces keep their value.  One thread
// per face: the pipe grids are small and the three stencil sources differ.
template <class T>
__global__ void k_eno3_pipe(T* comp, const T* __restrict__ gen, const T* __restrict__ gx, const T* __restrict__ gz,
                            const T* __restrict__ ug, const T* __restrict__ vg, const T* __restrict__ wg, Lay Lf,
                            Lay Lu, Lay Lv, Lay Lw, int axis, PipeGeom G, T h, T dt, int fi0, int fi1, int fk0,
                            int fk1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= Lf.nx || j >= Lf.ny || k >= Lf.nz) return;
  if ((i == fi0 || i == fi1) && (k == fk0 || k == fk1)) return;  // the fixed centre line
  if (!(pipe_wall_distance(G, 1 + axis, i, k) < 0.0)) return;
  const T inv = T(1) / h, o2 = T(0.5) / h, o3 = inv * T(1) / T(3);
  T vx[7], vy[7], vz[7];
#pragma unroll
  for (int q = 0; q < 7; ++q) {
    vx[q] = gx[Lf.at(i + q - 3, j, k)];
    vy[q] = gen[Lf.at(i, j + q - 3, k)];
    vz[q] = gz[Lf.at(i, j, k + q - 3)];
  }
  T uvel, vvel, wvel;
  mac_velocity(ug, vg, wg, Lu, Lv, Lw, axis, i, j, k, uvel, vvel, wvel);
  T dxm, dxp, dym, dyp, dzm, dzp;
  eno3_pair7(vx, h, inv, o2, o3, dxm, dxp);
  eno3_pair7(vy, h, inv, o2, o3, dym, dyp);
  eno3_pair7(vz, h, inv, o2, o3, dzm, dzp);
  const int64_t f = Lf.at(i, j, k);
  comp[f] = comp[f] - dt * ((uvel * (uvel > T(0) ? dxm : dxp) + vvel * (vvel > T(0) ? dym : dyp)) +
                            wvel * (wvel > T(0) ? dzm : dzp));
}

// ---------------------------------------------------------------------------
// Sussman reinitialisation
// ---------------------------------------------------------------------------

template <class T>
__global__ void k_sign(const T* __restrict__ phi, T* __restrict__ s, Lay L, T dx) {
  FS_IJK(L);
  const int64_t c = L.at(i, j, k);
  const T p = phi[c];
  s[c] = p / sqrt(p * p + dx * dx);
}

// Per-axis Godunov choice of the reference's case tree.  code: 0 D-, 1 D+,
// 2 dropped (expansion fan).
template <class T>
__device__ __forceinline__ T godunov(T s, T dm, T dp, int& code, bool& shock) {
  const T sm = s * dm, sp = s * dp;
  shock = false;
  if (sp >= T(0) && sm >= T(0)) { code = 0; return dm; }
  if (sp <= T(0) && sm <= T(0)) { code = 1; return dp; }
  if (sp > T(0) && sm < T(0)) { code = 2; return T(0); }
  shock = true;  // sp < 0 < sm
  const T ss = s * (fabs(dp) - fabs(dm)) / (dp - dm);
  if (ss > T(0)) { code = 0; return dm; }
  code = 1;
  return dp;
}

// One pseudo-step phi - dtau*S*(|grad phi|_G - 1) with the sign-preserving
// clamp; out = c0*base + c1*(that) when c0 != 0 (RK block combination).
template <class T>
__global__ void __launch_bounds__(kTX * kTY) k_sussman(const T* __restrict__ src, const T* __restrict__ sgn,
                                                    const T* __restrict__ base, T* __restrict__ out, Lay L, T inv_h,
                                                    T eps, T dtau, T c0, T c1, int typo, int kchunk) {
  __shared__ T ring[kRing * kRW * kRH];
  const int i0 = blockIdx.x * kTX, j0 = blockIdx.y * kTY;
  const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  const int k0 = blockIdx.z * kchunk, k1 = min(L.nz, k0 + kchunk);
  const bool valid = i < L.nx && j < L.ny;
  for (int kk = k0 - GH; kk < k0 + GH; ++kk) stage_plane(ring, src, L, i0, j0, kk);
  for (int k = k0; k < k1; ++k) {
    stage_plane(ring, src, L, i0, j0, k + GH);
    __syncthreads();
    if (valid) {
      const int64_t c = L.at(i, j, k);
      T vx[7], vy[7], vz[7];
      ring_samples(ring, k, vx, vy, vz);
      T dxm, dxp, dym, dyp, dzm, dzp;
      weno_pair7(vx, inv_h, eps, dxm, dxp);
      weno_pair7(vy, inv_h, eps, dym, dyp);
      weno_pair7(vz, inv_h, eps, dzm, dzp);
      const T s = sgn[c];
      int cx, cy, cz;
      bool shx, shy, shz;
      const T gx = godunov(s, dxm, dxp, cx, shx);
      const T gy = godunov(s, dym, dyp, cy, shy);
      const T gz = godunov(s, dzm, dzp, cz, shz);
      T mag = sqrt((gx * gx + gy * gy) + gz * gz) - T(1);
      if (typo && shx && shy && cy == 1 && cz == 2) mag = (sqrt(gx * gx) + gy * gy) - T(1);
      T r = vx[3] - dtau * s * mag;
      if (s * r < T(0)) {
        if (s < T(0)) r = -eps;
        if (s > T(0)) r = eps;
      }
      out[c] = c0 == T(0) ? r : c0 * base[c] + c1 * r;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// elementwise helpers
// ---------------------------------------------------------------------------

// out = a*x + b*y over the interior of layout L.
template <class T>
__global__ void k_axpby(T* __restrict__ out, const T* __restrict__ x, const T* __restrict__ y, T a, T b, Lay L) {
  FS_IJK(L);
  const int64_t c = L.at(i, j, k);
  out[c] = a * x[c] + b * y[c];
}

// Add a constant (gravity*dt) to every interior face except the two wall
// planes normal to the component (which hold the no-penetration zero).
template <class T>
__global__ void k_add_const_interior_faces(T* __restrict__ f, Lay L, int axis, T value, int skip_walls) {
  FS_IJK(L);
  if (skip_walls) {
    const int e = axis == 0 ? i : (axis == 1 ? j : k);
    const int n = axis == 0 ? L.nx : (axis == 1 ? L.ny : L.nz);
    if (e == 0 || e == n - 1) return;
  }
  f[L.at(i, j, k)] += value;
}

// Zero the two wall planes normal to a face component.
template <class T>
__global__ void k_zero_walls(T* __restrict__ f, Lay L, int axis) {
  FS_IJK(L);
  const int e = axis == 0 ? i : (axis == 1 ? j : k);
  const int n = axis == 0 ? L.nx : (axis == 1 ? L.ny : L.nz);
  if (e == 0 || e == n - 1) f[L.at(i, j, k)] = T(0);
}

// ---------------------------------------------------------------------------
// host wrappers
// ---------------------------------------------------------------------------

template <class T>
void weno5_levelset(const T* src, const T* base, T* out, const T* u, const T* v, const T* w, const Lay& L,
                    const Lay& Lu, const Lay& Lv, const Lay& Lw, double dx, double eps, double dt, double c0, double c1,
                    cudaStream_t s, const PipeGeom* pipe) {
  const StagedGrid g = staged_grid(L);
  PipeGeom none{};
  k_weno5_levelset<T><<<g.grid, dim3(kTX, kTY, 1), 0, s>>>(src, base, out, u, v, w, L, Lu, Lv, Lw, T(1.0 / dx),
                                                           T(eps), T(dt), T(c0), T(c1), g.kchunk,
                                                           pipe ? *pipe : none);
}

template <class T>
void weno5_mac(const T* comp, T* out, const T* u, const T* v, const T* w, const Lay& Lc, const Lay& Lu, const Lay& Lv,
               const Lay& Lw, int axis, double dx, double eps, double dt, cudaStream_t s) {
  const StagedGrid g = staged_grid(Lc);
  k_weno5_mac<T><<<g.grid, dim3(kTX, kTY, 1), 0, s>>>(comp, out, u, v, w, Lc, Lu, Lv, Lw, axis, T(1.0 / dx), T(eps),
                                                      T(dt), g.kchunk);
}

template <class T>
void eno3_mac(const T* comp, T* out, const T* u, const T* v, const T* w, const Lay& Lc, const Lay& Lu, const Lay& Lv,
              const Lay& Lw, int axis, double dx, double dt, cudaStream_t s) {
  const StagedGrid g = staged_grid(Lc);
  k_eno3_mac<T><<<g.grid, dim3(kTX, kTY, 1), 0, s>>>(comp, out, u, v, w, Lc, Lu, Lv, Lw, axis, T(dx), T(dt),
                                                     g.kchunk);
}

template <class T>
void eno3_pipe(T* comp, const T* gen, const T* gx, const T* gz, const T* ug, const T* vg, const T* wg, const Lay& Lc,
               const Lay& Lu, const Lay& Lv, const Lay& Lw, int axis, const PipeGeom& G, double dx, double dt,
               cudaStream_t s) {
  const Lay& Lf = axis == 0 ? Lu : axis == 1 ? Lv : Lw;
  // the faces Solve_Velocity holds fixed (ADVECTION_3D.h:246-275): the
  // integer halves of the face grid's last indices
  int fi0, fi1, fk0, fk1;
  if (axis == 0) { fi0 = (Lf.nx - 1) / 2; fi1 = fi0 + 1; fk0 = fk1 = (Lc.nz - 1) / 2; }
  else if (axis == 1) { fi0 = fi1 = (Lc.nx - 1) / 2; fk0 = fk1 = (Lc.nz - 1) / 2; }
  else { fi0 = fi1 = (Lc.nx - 1) / 2; fk0 = (Lf.nz - 1) / 2; fk1 = fk0 + 1; }
  Launch3 g = launch3(Lf.nx, Lf.ny, Lf.nz);
  k_eno3_pipe<T><<<g.grid, g.block, 0, s>>>(comp, gen, gx, gz, ug, vg, wg, Lf, Lu, Lv, Lw, axis, G, T(dx), T(dt), fi0,
                                            fi1, fk0, fk1);
}

template <class T>
void sign_function(const T* phi, T* sgn, const Lay& L, double dx, cudaStream_t s) {
  Launch3 g = launch3(L.nx, L.ny, L.nz);
  k_sign<T><<<g.grid, g.block, 0, s>>>(phi, sgn, L, T(dx));
}

template <class T>
void sussman_step(const T* src, const T* sgn, const T* base, T* out, const Lay& L, double dx, double eps, double dtau,
                  double c0, double c1, int typo, cudaStream_t s) {
  const StagedGrid g = staged_grid(L);
  k_sussman<T><<<g.grid, dim3(kTX, kTY, 1), 0, s>>>(src, sgn, base, out, L, T(1.0 / dx), T(eps), T(dtau), T(c0),
                                                    T(c1), typo, g.kchunk);
}

template <class T>
void axpby(T* out, const T* x, const T* y, double a, double b, const Lay& L, cudaStream_t s) {
  Launch3 g = launch3(L.nx, L.ny, L.nz);
  k_axpby<T><<<g.grid, g.block, 0, s>>>(out, x, y, T(a), T(b), L);
}

template <class T>
void add_const_faces(T* f, const Lay& L, int axis, double value, int skip_walls, cudaStream_t s) {
  Launch3 g = launch3(L.nx, L.ny, L.nz);
  k_add_const_interior_faces<T><<<g.grid, g.block, 0, s>>>(f, L, axis, T(value), skip_walls);
}

template <class T>
void zero_walls(T* f, const Lay& L, int axis, cudaStream_t s) {
  Launch3 g = launch3(L.nx, L.ny, L.nz);
  k_zero_walls<T><<<g.grid, g.block, 0, s>>>(f, L, axis);
}

#define FS_INST(T)                                                                                                    \
  template void fill_extrap<T>(T*, const Lay&, cudaStream_t);                                                         \
  template void weno5_levelset<T>(const T*, const T*, T*, const T*, const T*, const T*, const Lay&, const Lay&,       \
                                  const Lay&, const Lay&, double, double, double, double, double, cudaStream_t,       \
                                  const PipeGeom*);                                                                   \
  template void weno5_mac<T>(const T*, T*, const T*, const T*, const T*, const Lay&, const Lay&, const Lay&,          \
                             const Lay&, int, double, double, double, cudaStream_t);                                  \
  template void eno3_pipe<T>(T*, const T*, const T*, const T*, const T*, const T*, const T*, const Lay&, const Lay&,  \
                             const Lay&, const Lay&, int, const PipeGeom&, double, double, cudaStream_t);             \
  template void eno3_mac<T>(const T*, T*, const T*, const T*, const T*, const Lay&, const Lay&, const Lay&,           \
                            const Lay&, int, double, double, cudaStream_t);                                          \
  template void sign_function<T>(const T*, T*, const Lay&, double, cudaStream_t);                                    \
  template void sussman_step<T>(const T*, const T*, const T*, T*, const Lay&, double, double, double, double, double, \
                                int, cudaStream_t);                                                                   \
  template void axpby<T>(T*, const T*, const T*, double, double, const Lay&, cudaStream_t);                          \
  template void add_const_faces<T>(T*, const Lay&, int, double, int, cudaStream_t);                                  \
  template void zero_walls<T>(T*, const Lay&, int, cudaStream_t);

FS_INST(float)
FS_INST(double)

}  // namespace fsb
