// Jacobi-preconditioned conjugate gradients on a matrix-free seven-point
// operator (PCG_METHOD.cpp:4-126 restated for the GPU), with optional
// reliable updates for the mixed-precision pressure solve.
//
// Vector types: V for the operator, the residual r, the search direction p
// and q = A p; X for the iterate x.  V = X = double is the FP64 path,
// V = X = float the viscosity solves in FP32 storage, and V = float,
// X = double the mixed-precision pressure solve, whose iterate is the FP64
// pressure itself.  The scalars (alpha, beta, r.z, r.r) are FP64 always.
//
// One iteration is three kernels (details at k_cg_spmv below):
//   spmv    q = A p, p.q, alpha                (reads p, ax, ay, az; writes q)
//   update  r -= alpha q, r.z, r.r, beta       (reads r, q, diag; writes r)
//   pupdate x += alpha p, p = r/diag + beta p  (reads x, p, r, diag; writes x, p)
// z = r/diag is never stored: 64 bytes per unknown and iteration with FP32
// vectors, an FP64 iterate and the bf16 inverse diagonal (Op7::dinv16), 120
// in FP64.  Dot products are reduced in
// FP64 per block and finished by the last block (deterministic for a given
// grid), which also takes the scalar decisions (alpha, beta, convergence,
// caps, breakdown) and writes them to the PcgState in device memory.  Every
// kernel starts by reading `done`, so iterations captured in a CUDA graph
// cost microseconds once a solve stops.
//
// Reliable updates (Clark et al., "Solving lattice QCD systems of equations
// using mixed precision solvers on GPUs", 2010): in the FP32 pressure solve
// the update kernel pauses the iteration (done = 2) whenever the recursive
// residual has dropped by `reliable_delta` since the last true residual; the
// host then recomputes the true residual of the FP64 pressure in FP64 and
// resumes the same Krylov iteration (pcg_resume) with that residual, keeping
// the search direction.  The FP32 iteration therefore converges like
// one long CG instead of a sequence of restarted ones.
#include <algorithm>
#include <cstdlib>

#include "fs_kernels.h"

namespace fsb {

static int g_sm_count = 0;
constexpr int g_blocks_per_sm = 6;  // 6 x 256 threads: fully resident for kernels up to 40 registers

int reduction_blocks(int64_t n) {
  if (g_sm_count <= 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) g_sm_count = 148;
  }
  const int64_t want = (n + kRedThreads - 1) / kRedThreads;
  const int64_t cap = (int64_t)g_blocks_per_sm * g_sm_count;
  return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

int pcg_blocks(const Lay& L) { return reduction_blocks((int64_t)L.nx * L.ny * L.nz); }

// The Jacobi preconditioner z = M^-1 r: r / diag, or r * dinv16 when the
// operator carries the bf16 inverse diagonal (Op7::dinv16).
__device__ __forceinline__ float bf16_to_float(unsigned short b) { return __uint_as_float((unsigned)b << 16); }
template <class V, class R>
__device__ __forceinline__ R precond1(const Op7<V>& A, R r, int64_t c) {
  return A.dinv16 ? r * (R)bf16_to_float(A.dinv16[c]) : r / (R)A.diag[c];
}

// (A x)_c evaluated in the type X of x (the operator's coefficients are
// converted): FP32 iterates get FP32 arithmetic, FP64 iterates FP64.
// The flux form is evaluated here in FP64 (loads in their storage type):
// for smooth x the six fluxes nearly cancel, and FP64 keeps q exact to
// rounding.  (The iteration's own SpMV, k_cg_spmv, may form FP32 fluxes in
// FP32: see Op7::flux32.)
template <class V, class X>
__device__ __forceinline__ X apply7(const Op7<V>& A, const X* __restrict__ x, int64_t c) {
  const int64_t sy = A.L.px, sz = A.L.slab;
  const X xc = x[c];
  if (A.flux_form) {
    const double d = (double)xc;
    double acc = (double)A.ax[c] * (d - (double)x[c - 1]) + (double)A.ax[c + 1] * (d - (double)x[c + 1]);
    acc += (double)A.ay[c] * (d - (double)x[c - sy]) + (double)A.ay[c + sy] * (d - (double)x[c + sy]);
    acc += (double)A.az[c] * (d - (double)x[c - sz]) + (double)A.az[c + sz] * (d - (double)x[c + sz]);
    if (c == (A.c_extra >= 0 ? A.c_extra : A.L.at(0, 0, 0))) acc += (*A.extra0) * d;
    return (X)acc;
  }
  X acc = (X)A.diag[c] * xc;
  acc -= (X)A.ax[c] * x[c - 1] + (X)A.ax[c + 1] * x[c + 1];
  acc -= (X)A.ay[c] * x[c - sy] + (X)A.ay[c + sy] * x[c + sy];
  acc -= (X)A.az[c] * x[c - sz] + (X)A.az[c + sz] * x[c + sz];
  return acc;
}

// Three FP64 sums through one grid reduction (1-D grids).
__device__ __forceinline__ bool grid_reduce3(double a, double b, double c, double* partials, unsigned int* ticket,
                                             double out[3]) {
  __shared__ bool is_last;
  __shared__ double tot[3];
  a = block_sum(a);
  __syncthreads();
  b = block_sum(b);
  __syncthreads();
  c = block_sum(c);
  const int nb = gridDim.x;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = a;
    partials[nb + blockIdx.x] = b;
    partials[2 * nb + blockIdx.x] = c;
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    is_last = (t == (unsigned int)(nb - 1));
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  for (int m = 0; m < 3; ++m) {
    double s = 0.0;
#pragma unroll 8
    for (int q = threadIdx.x; q < nb; q += blockDim.x) s += __ldcg(partials + m * nb + q);  // as in grid_reduce_sum
    s = block_sum(s);
    if (threadIdx.x == 0) tot[m] = s;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = tot[0];
    out[1] = tot[1];
    out[2] = tot[2];
    *ticket = 0u;
  }
  return threadIdx.x == 0;
}

__device__ __forceinline__ bool stop_test(const PcgState* st, double rz, double rr) {
  switch (st->criterion) {
    case 1: return rz < st->tol * st->tol;                 // the reference's r.z < tol^2
    case 2: return rr < st->tol * st->tol;                 // absolute 2-norm
    default: return sqrt(rr) <= st->tol * sqrt(st->bb);    // relative 2-norm
  }
}

template <class V, class RT>
__global__ void __launch_bounds__(kRedThreads) k_pcg_init(Op7<V> A, const RT* b, RT* x, RT* r, V* __restrict__ p,
                                                          PcgState* st, double* partials) {
  double rz = 0.0, rr = 0.0, bb = 0.0;
  Cursor cur;
  for (cur.init(A.L); cur.valid(A.L); cur.next(A.L)) {
    const int64_t c = A.L.at(cur.i, cur.j, cur.k);
    const RT bv = b[c];
    const RT rv = bv - apply7<V, RT>(A, x, c);
    const RT z = precond1<V, RT>(A, rv, c);
    r[c] = rv;  // b may alias r: each element is read before it is written
    p[c] = (V)z;
    rz += (double)rv * (double)z;
    rr += (double)rv * (double)rv;
    bb += (double)bv * (double)bv;
  }
  double tot[3];
  if (grid_reduce3(rz, rr, bb, partials, &st->ticket, tot)) {
    st->rz = tot[0];
    st->rr = tot[1];
    st->bb = tot[2];
    st->iter = 0;
    st->beta = 0.0;
    st->best_rr = tot[1];
    st->max_rr = tot[1];
    st->rz_prev = tot[0];
    st->stall = 0;
    st->status = PCG_RUNNING;
    st->done = 0;
    if (!isfinite(tot[0]) || !isfinite(tot[1])) {
      st->status = PCG_NONFINITE;
      st->done = 1;
    } else if (tot[2] == 0.0 || tot[1] == 0.0 || (st->criterion != 1 && stop_test(st, tot[0], tot[1]))) {
      // zero right-hand side or an initial guess that already satisfies the test
      st->status = PCG_CONVERGED;
      st->done = 1;
    } else if (st->max_iter <= 0) {
      st->status = PCG_MAXITER;
      st->done = 1;
    }
  }
}

template <class V, class RT>
__global__ void __launch_bounds__(kRedThreads) k_pcg_pupdate(Op7<V> A, const RT* __restrict__ r, V* __restrict__ p,
                                                             PcgState* st) {
  if (((volatile PcgState*)st)->done) return;
  const RT beta = (RT)((volatile PcgState*)st)->beta;
  Cursor cur;
  for (cur.init(A.L); cur.valid(A.L); cur.next(A.L)) {
    const int64_t c = A.L.at(cur.i, cur.j, cur.k);
    p[c] = (V)((RT)p[c] * beta + precond1<V, RT>(A, r[c], c));
  }
}

// After the caller replaced r by the true residual: r.z and r.r of the new
// residual, beta for the direction update (0 on a restart), and the
// iteration resumes (done = 0).
template <class V, class RT>
__global__ void __launch_bounds__(kRedThreads) k_pcg_resume(Op7<V> A, const RT* __restrict__ r, PcgState* st,
                                                            double* partials, int restart) {
  double rz = 0.0, rr = 0.0;
  Cursor cur;
  for (cur.init(A.L); cur.valid(A.L); cur.next(A.L)) {
    const int64_t c = A.L.at(cur.i, cur.j, cur.k);
    const RT rv = r[c];
    rz += (double)rv * (double)precond1<V, RT>(A, rv, c);
    rr += (double)rv * (double)rv;
  }
  double tot[3];
  if (grid_reduce3(rz, rr, 0.0, partials, &st->ticket, tot)) {
    // the direction update continues from the last accepted step: beta
    // relates the new r.z to the r.z that step started from
    st->beta = restart ? 0.0 : tot[0] / st->rz_prev;
    st->rz = tot[0];
    st->rr = tot[1];
    st->max_rr = tot[1];
    st->best_rr = tot[1];
    st->stall = 0;
    st->status = PCG_RUNNING;
    st->done = 0;
    if (!isfinite(tot[0]) || !isfinite(tot[1])) {
      st->status = PCG_NONFINITE;
      st->done = 1;
    }
  }
}

template <class V, class RT>
void pcg_init(const Op7<V>& A, const RT* b, RT* x, RT* r, V* p, PcgState* st, double* partials, cudaStream_t s) {
  k_pcg_init<V, RT><<<pcg_blocks(A.L), kRedThreads, 0, s>>>(A, b, x, r, p, st, partials);
}

template <class V, class RT>
void pcg_resume(const Op7<V>& A, const RT* r, V* p, PcgState* st, double* partials, int restart, cudaStream_t s) {
  const int nb = pcg_blocks(A.L);
  k_pcg_resume<V, RT><<<nb, kRedThreads, 0, s>>>(A, r, st, partials, restart);
  k_pcg_pupdate<V, RT><<<nb, kRedThreads, 0, s>>>(A, r, p, st);
}

// ---------------------------------------------------------------------------
// The iteration with a deferred iterate update.
//
// The iterate is touched once per iteration, in the direction update that
// reads p anyway, so the residual update streams neither p nor x.  When an
// iteration stops in the residual update (converged, capped, paused for a
// reliable update) the direction update still applies the pending
// x += alpha p and leaves p alone; x_pending is cleared by the last block of
// the direction update so that later launches of a captured batch do not
// apply it twice.
//
// In the pressure solve the iterate must stay FP64: FP32 rounding of x is
// amplified by ||A|| ||x|| / ||b||, which is of the order of the condition
// number at density ratio 1000.  FP32 rounding of r and q only perturbs the
// recursion by eps32 ||r|| per step (reliable updates bound what
// accumulates), and FP32 rounding of p is harmless because q is computed
// from the rounded p itself.
// ---------------------------------------------------------------------------

// ---- four-cell vectors along x (rows start 16/32-byte aligned, see Lay)
template <class T> struct V4 { T a, b, c, d; };

__device__ __forceinline__ V4<float> ld4(const float* p) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ V4<double> ld4(const double* p) {
  const double2 v0 = reinterpret_cast<const double2*>(p)[0];
  const double2 v1 = reinterpret_cast<const double2*>(p)[1];
  return {v0.x, v0.y, v1.x, v1.y};
}
// stores the lanes below `valid` (4: one vector store)
__device__ __forceinline__ void st4(float* p, const V4<float>& v, int valid) {
  if (valid >= 4) {
    *reinterpret_cast<float4*>(p) = make_float4(v.a, v.b, v.c, v.d);
  } else {
    if (valid > 0) p[0] = v.a;
    if (valid > 1) p[1] = v.b;
    if (valid > 2) p[2] = v.c;
  }
}
__device__ __forceinline__ void st4(double* p, const V4<double>& v, int valid) {
  if (valid >= 4) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v.a, v.b);
    reinterpret_cast<double2*>(p)[1] = make_double2(v.c, v.d);
  } else {
    if (valid > 0) p[0] = v.a;
    if (valid > 1) p[1] = v.b;
    if (valid > 2) p[2] = v.c;
  }
}
template <class T> __device__ __forceinline__ T lane(const V4<T>& v, int m) {
  return m == 0 ? v.a : (m == 1 ? v.b : (m == 2 ? v.c : v.d));
}
template <class T> __device__ __forceinline__ void set_lane(V4<T>& v, int m, T x) {
  if (m == 0) v.a = x; else if (m == 1) v.b = x; else if (m == 2) v.c = x; else v.d = x;
}

// ---- the Jacobi preconditioner z = M^-1 r on four cells (precond1 above)
template <class V>
__device__ __forceinline__ V4<V> precond4(const Op7<V>& A, const V4<V>& r, int64_t c) {
  if (A.dinv16) {
    const uint2 u = *reinterpret_cast<const uint2*>(A.dinv16 + c);  // 4 bf16, 8-byte aligned (c % 4 == 0)
    return {r.a * (V)__uint_as_float(u.x << 16), r.b * (V)__uint_as_float(u.x & 0xffff0000u),
            r.c * (V)__uint_as_float(u.y << 16), r.d * (V)__uint_as_float(u.y & 0xffff0000u)};
  }
  const V4<V> d = ld4(A.diag + c);
  return {r.a / d.a, r.b / d.b, r.c / d.c, r.d / d.d};
}

// Grid-stride cursor over (vector, j, k): vector w covers i = 4w .. 4w+3.
struct VecCursor {
  Lay Lv;  // the layout with nx replaced by the number of vectors per row
  Cursor cur;
  __device__ __forceinline__ void init(const Lay& L) {
    Lv = L;
    Lv.nx = (L.nx + 3) >> 2;
    cur.init(Lv);
  }
  __device__ __forceinline__ bool valid() const { return cur.valid(Lv); }
  __device__ __forceinline__ void next() { cur.next(Lv); }
};

// ---- SpMV: q = A p with the p.q reduction and the step length.
//
// One thread owns four consecutive cells of a row (i = 4w .. 4w+3, j) and
// marches up a chunk of planes k0 .. k1-1.  The z neighbours of p and the
// upper z coupling stay in registers from one plane to the next (each plane
// of p and az is loaded once), the x neighbours come from the adjacent lanes
// of the warp by shuffle (global loads only at the two ends of a warp or of
// a row) and the y neighbours are rows that the neighbouring threads of the
// block load in the same plane (L1 hits).  Blocks are 32 x 8 threads
// (128 x 8 cells); the grid is the xy tiles times as many z chunks as fill
// the resident blocks of the GPU.
template <class V>
__device__ __forceinline__ void spmv_row4(const Op7<V>& A, const V* __restrict__ p, int64_t c, int i0,
                                          const V4<V>& pc, const V4<V>& pdn, const V4<V>& pup, const V4<V>& azc,
                                          const V4<V>& azu, V4<V>& q) {
  const int64_t sy = A.L.px;
  const int lane_id = threadIdx.x & 31;
  const V4<V> ps = ld4(p + c - sy), pn = ld4(p + c + sy);
  const V4<V> ayc = ld4(A.ay + c), ayn = ld4(A.ay + c + sy);
  const V4<V> axc = ld4(A.ax + c);
  // x neighbours: p[i0-1], p[i0+4] and ax[i0+4] from the adjacent lanes
  V pl = __shfl_up_sync(0xffffffffu, pc.d, 1);
  V pr = __shfl_down_sync(0xffffffffu, pc.a, 1);
  V axr = __shfl_down_sync(0xffffffffu, axc.a, 1);
  if (lane_id == 0) pl = p[c - 1];
  if (lane_id == 31 || i0 + 4 >= A.L.nx) {  // warp end, or the row ends in this vector
    pr = p[c + 4];
    axr = A.ax[c + 4];
  }
  const int64_t c00 = A.c_extra >= 0 ? A.c_extra : A.L.at(0, 0, 0);
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const V xc = lane(pc, m);
    const V xl = m == 0 ? pl : lane(pc, m - 1);
    const V xr = m == 3 ? pr : lane(pc, m + 1);
    const V ar = m == 3 ? axr : lane(axc, m + 1);
    V out;
    if (A.flux_form && A.flux32 == 2) {
      V acc = lane(axc, m) * (xc - xl) + ar * (xc - xr);
      acc += lane(ayc, m) * (xc - lane(ps, m)) + lane(ayn, m) * (xc - lane(pn, m));
      acc += lane(azc, m) * (xc - lane(pdn, m)) + lane(azu, m) * (xc - lane(pup, m));
      if (c + m == c00) acc += (V)(*A.extra0) * xc;
      out = acc;
    } else if (A.flux_form && A.flux32 == 1) {
      double acc = (double)(lane(axc, m) * (xc - xl)) + (double)(ar * (xc - xr));
      acc += (double)(lane(ayc, m) * (xc - lane(ps, m))) + (double)(lane(ayn, m) * (xc - lane(pn, m)));
      acc += (double)(lane(azc, m) * (xc - lane(pdn, m))) + (double)(lane(azu, m) * (xc - lane(pup, m)));
      if (c + m == c00) acc += (*A.extra0) * (double)xc;
      out = (V)acc;
    } else if (A.flux_form) {
      // flux form in FP64 arithmetic (see apply7)
      const double d = (double)xc;
      double acc = (double)lane(axc, m) * (d - (double)xl) + (double)ar * (d - (double)xr);
      acc += (double)lane(ayc, m) * (d - (double)lane(ps, m)) + (double)lane(ayn, m) * (d - (double)lane(pn, m));
      acc += (double)lane(azc, m) * (d - (double)lane(pdn, m)) + (double)lane(azu, m) * (d - (double)lane(pup, m));
      if (c + m == c00) acc += (*A.extra0) * d;
      out = (V)acc;
    } else {
      V acc = A.diag[c + m] * xc;
      acc -= lane(axc, m) * xl + ar * xr;
      acc -= lane(ayc, m) * lane(ps, m) + lane(ayn, m) * lane(pn, m);
      acc -= lane(azc, m) * lane(pdn, m) + lane(azu, m) * lane(pup, m);
      out = acc;
    }
    set_lane(q, m, out);
  }
}

// p.q over the grid and the step length alpha = r.z / p.q (last block).
__device__ __forceinline__ void spmv_alpha(double pq, PcgState* st, double* partials) {
  pq = block_sum(pq);
  double tot;
  if (grid_reduce_sum(pq, partials, &st->ticket, &tot)) {
    st->pq = tot;
    const double alpha = st->rz / tot;
    if (!(tot > 0.0) || !isfinite(alpha)) {
      // a non-positive p.Ap (or an infinite step): the iteration has lost its
      // footing in this arithmetic; keep the iterate and stop
      st->status = PCG_STAGNATED;
      st->done = 1;
      st->x_pending = 0;
    } else {
      st->alpha = alpha;
      st->x_pending = 1;
    }
  }
}

template <class V, int MINB>
__global__ void __launch_bounds__(256, MINB) k_cg_spmv(Op7<V> A, const V* __restrict__ p, V* __restrict__ q,
                                                 PcgState* st, double* partials, int kchunk) {
  if (((volatile PcgState*)st)->done) return;
  const Lay& L = A.L;
  const int w = blockIdx.x * 32 + threadIdx.x;  // vector index along x
  const int j = blockIdx.y * 8 + threadIdx.y;
  const int i0 = 4 * w;
  const int k0 = blockIdx.z * kchunk;
  const int k1 = min(L.nz, k0 + kchunk);
  // threads past the end of a row or of the box compute on a clamped row and
  // store nothing; every thread of the warp takes part in the shuffles
  const bool row_ok = j < L.ny && i0 < L.nx;
  const int nvalid = row_ok ? min(4, L.nx - i0) : 0;
  const int jj = min(j, L.ny - 1), ii = min(i0, 4 * ((L.nx - 1) >> 2));
  const int64_t sz = L.slab;
  double pq = 0.0;
  if (k0 < k1) {
    int64_t c = L.at(ii, jj, k0);
    V4<V> pdn = ld4(p + c - sz), pc = ld4(p + c), azc = ld4(A.az + c);
#pragma unroll 2
    for (int k = k0; k < k1; ++k, c += sz) {
      const V4<V> pup = ld4(p + c + sz), azu = ld4(A.az + c + sz);
      V4<V> qv;
      spmv_row4<V>(A, p, c, ii, pc, pdn, pup, azc, azu, qv);
      if (nvalid > 0) {
        st4(q + c, qv, nvalid);
        pq += (double)pc.a * (double)qv.a;  // p.q of the stored q, as the residual update uses it
        if (nvalid > 1) pq += (double)pc.b * (double)qv.b;
        if (nvalid > 2) pq += (double)pc.c * (double)qv.c;
        if (nvalid > 3) pq += (double)pc.d * (double)qv.d;
      }
      pdn = pc;
      pc = pup;
      azc = azu;
    }
  }
  spmv_alpha(pq, st, partials);
}

// ---- p.q and the step length of a SpMV that does not reduce (the
// red-black black pass): one streaming pass over p and q, FP64 products
// summed per thread, per block and by the last block, which takes the same
// decisions as spmv_alpha.  Measured at 256^3 on the packed black vectors:
// the black pass without its reduction plus this pass take 88 us against 98
// us for the black pass reducing p.q itself (its per-thread accumulation
// across the planes of a chunk held back the loads of the next plane).
template <class V>
__global__ void __launch_bounds__(kRedThreads) k_pq_alpha(Op7<V> A, const V* __restrict__ p, const V* __restrict__ q,
                                                          PcgState* st, double* partials) {
  if (((volatile PcgState*)st)->done) return;
  double pq = 0.0;
  VecCursor vc;
  for (vc.init(A.L); vc.valid(); vc.next()) {
    const int i0 = 4 * vc.cur.i;
    const int64_t c = A.L.at(i0, vc.cur.j, vc.cur.k);
    const int nvalid = min(4, A.L.nx - i0);
    const V4<V> pv = ld4(p + c), qv = ld4(q + c);
#pragma unroll
    for (int m = 0; m < 4; ++m)
      if (m < nvalid) pq += (double)lane(pv, m) * (double)lane(qv, m);
  }
  spmv_alpha(pq, st, partials);
}

// ---- residual update: r -= alpha q, r.z and r.r, beta and the decisions
template <class V>
__global__ void __launch_bounds__(kRedThreads) k_cg_update(Op7<V> A, V* __restrict__ r, const V* __restrict__ q,
                                                           PcgState* st, double* partials) {
  if (((volatile PcgState*)st)->done) return;
  const V alpha = (V)((volatile PcgState*)st)->alpha;
  double rz = 0.0, rr = 0.0;
  VecCursor vc;
  for (vc.init(A.L); vc.valid(); vc.next()) {
    const int i0 = 4 * vc.cur.i;
    const int64_t c = A.L.at(i0, vc.cur.j, vc.cur.k);
    const int nvalid = min(4, A.L.nx - i0);
    V4<V> rv = ld4(r + c);
    const V4<V> qv = ld4(q + c);
    rv.a -= alpha * qv.a;
    rv.b -= alpha * qv.b;
    rv.c -= alpha * qv.c;
    rv.d -= alpha * qv.d;
    st4(r + c, rv, nvalid);
    // r.z and r.r of the vector's cells in the vector type (z formed as the
    // direction update forms it), accumulated in FP64 across vectors
    const V4<V> zv = precond4(A, rv, c);
    V rz4 = V(0), rr4 = V(0);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      if (m < nvalid) {
        const V rm = lane(rv, m);
        rz4 += rm * lane(zv, m);
        rr4 += rm * rm;
      }
    }
    rz += (double)rz4;
    rr += (double)rr4;
  }
  double tot[3];
  if (grid_reduce3(rz, rr, 0.0, partials, &st->ticket, tot)) {
    const double rz_old = st->rz;
    st->rr = tot[1];
    st->rz_prev = rz_old;
    st->rz = tot[0];
    if (tot[1] < 0.99 * st->best_rr) {
      st->best_rr = tot[1];
      st->stall = 0;
    } else {
      st->stall += 1;
    }
    if (!isfinite(tot[0]) || !isfinite(tot[1])) {
      st->status = PCG_NONFINITE;
      st->done = 1;
      st->x_pending = 0;  // do not move the iterate along a step that produced non-finite values
    } else if (stop_test(st, tot[0], tot[1])) {
      st->status = PCG_CONVERGED;
      st->done = 1;
    } else {
      st->beta = tot[0] / rz_old;
      st->iter += 1;
      if (st->iter >= st->max_iter) {
        st->status = PCG_MAXITER;
        st->done = 1;
      } else if (st->stall_limit > 0 && st->stall >= st->stall_limit) {
        st->status = PCG_STAGNATED;
        st->done = 1;
      } else if (st->reliable_delta > 0.0 && tot[1] < st->reliable_delta * st->reliable_delta * st->max_rr) {
        st->status = PCG_RELIABLE_UPDATE;  // pause before the direction update
        st->done = 2;
      }
    }
  }
}

// ---- direction update: x += alpha p (when pending), p = r/diag + beta p
template <class V, class X>
__global__ void __launch_bounds__(kRedThreads) k_cg_pupdate(Op7<V> A, X* __restrict__ x, const V* __restrict__ r,
                                                            V* __restrict__ p, PcgState* st) {
  const volatile PcgState* vs = (volatile PcgState*)st;
  const bool move_x = vs->x_pending != 0;
  const bool move_p = vs->done == 0;
  if (!move_x && !move_p) return;  // uniform: every block reads the same state
  const double alpha = vs->alpha;
  const V beta = (V)vs->beta;
  VecCursor vc;
  for (vc.init(A.L); vc.valid(); vc.next()) {
    const int i0 = 4 * vc.cur.i;
    const int64_t c = A.L.at(i0, vc.cur.j, vc.cur.k);
    const int nvalid = min(4, A.L.nx - i0);
    V4<V> pv = ld4(p + c);
    if (move_x) {
      V4<X> xv = ld4(x + c);
      xv.a += (X)(alpha * (double)pv.a);
      xv.b += (X)(alpha * (double)pv.b);
      xv.c += (X)(alpha * (double)pv.c);
      xv.d += (X)(alpha * (double)pv.d);
      st4(x + c, xv, nvalid);
    }
    if (move_p) {
      const V4<V> zv = precond4(A, ld4(r + c), c);
      pv.a = pv.a * beta + zv.a;
      pv.b = pv.b * beta + zv.b;
      pv.c = pv.c * beta + zv.c;
      pv.d = pv.d * beta + zv.d;
      st4(p + c, pv, nvalid);
    }
  }
  if (move_x) {
    // every thread of this block has read x_pending before it is counted
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned int t = atomicAdd(&st->ticket2, 1u);
      if (t == gridDim.x - 1) {
        st->x_pending = 0;
        st->ticket2 = 0u;
      }
    }
  }
}

namespace {
int g_cg_blocks[2][2][3];  // [X double?][V double?][spmv, update, pupdate]: resident blocks per SM
// SpMV blocks per SM the compiler must fit; measured best at 256^3 (sweeps
// of 2, 3 and 4): 4 for FP32 vectors (64 registers, no spills to speak
// of), 2 for FP64 (128 registers; fewer spill)
template <class V> constexpr int spmv_minb() { return sizeof(V) == 4 ? 4 : 2; }
}  // namespace

template <class V, class X>
void cg_prepare() {
  reduction_blocks(1);  // SM count
  int* slot = g_cg_blocks[sizeof(X) == 8][sizeof(V) == 8];
  const void* spmv = (const void*)k_cg_spmv<V, spmv_minb<V>()>;
  const void* ks[3] = {spmv, (const void*)k_cg_update<V>, (const void*)k_cg_pupdate<V, X>};
  for (int m = 0; m < 3; ++m) {
    if (slot[m]) continue;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ks[m], 256, 0) != cudaSuccess || nb <= 0) nb = 1;
    slot[m] = std::min(nb, g_blocks_per_sm);
  }
}

int cg_max_blocks(const Lay& L) {
  const int tiles = ((L.nx + 127) / 128) * ((L.ny + 7) / 8);
  return std::max(tiles, reduction_blocks((int64_t)1 << 40));  // the resident-block cap
}

template <class V, class X>
void cg_iteration(const Op7<V>& A, X* x, V* r, V* p, V* q, PcgState* st, double* partials, cudaStream_t s) {
  const int* slot = g_cg_blocks[sizeof(X) == 8][sizeof(V) == 8];
  const Lay& L = A.L;
  // SpMV grid: xy tiles of 128 x 8 cells times z chunks filling the resident blocks
  const int tx = (L.nx + 127) / 128, ty = (L.ny + 7) / 8;
  const int want = std::max(1, slot[0]) * g_sm_count;
  const int chunks = std::max(1, std::min(L.nz, want / (tx * ty)));
  const int kchunk = (L.nz + chunks - 1) / chunks;
  const dim3 sg(tx, ty, (L.nz + kchunk - 1) / kchunk);
  k_cg_spmv<V, spmv_minb<V>()><<<sg, dim3(32, 8, 1), 0, s>>>(A, p, q, st, partials, kchunk);
  cg_vector_updates<V, X>(A, x, r, p, q, st, partials, s);
}

template <class V, class X>
void cg_vector_updates(const Op7<V>& A, X* x, V* r, V* p, V* q, PcgState* st, double* partials, cudaStream_t s) {
  const int* slot = g_cg_blocks[sizeof(X) == 8][sizeof(V) == 8];
  const Lay& L = A.L;
  // pointwise kernels: grid-stride over the vectors, resident blocks only
  const int64_t nvec = (int64_t)((L.nx + 3) >> 2) * L.ny * L.nz;
  auto grid = [&](int per_sm) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((nvec + kRedThreads - 1) / kRedThreads,
                                                       (int64_t)std::max(per_sm, 1) * g_sm_count));
  };
  k_cg_update<V><<<grid(slot[1]), kRedThreads, 0, s>>>(A, r, q, st, partials);
  // the direction update on two waves of blocks: measured at 256^3 on the
  // packed black vectors, 48 us against 56 us on one wave (fewer vectors per
  // thread, the second wave fills the first one's tail)
  k_cg_pupdate<V, X><<<grid(2 * slot[2]), kRedThreads, 0, s>>>(A, x, r, p, st);
}

template <class V>
void pq_alpha(const Op7<V>& A, const V* p, const V* q, PcgState* st, double* partials, cudaStream_t s) {
  const Lay& L = A.L;
  const int64_t nvec = (int64_t)((L.nx + 3) >> 2) * L.ny * L.nz;
  const int g = (int)std::max<int64_t>(1, std::min<int64_t>((nvec + kRedThreads - 1) / kRedThreads,
                                                            (int64_t)g_blocks_per_sm * g_sm_count));
  k_pq_alpha<V><<<g, kRedThreads, 0, s>>>(A, p, q, st, partials);
}
template void pq_alpha<float>(const Op7<float>&, const float*, const float*, PcgState*, double*, cudaStream_t);

template void cg_prepare<float, double>();
template void cg_prepare<double, double>();
template void cg_prepare<float, float>();
template void cg_iteration<float, double>(const Op7<float>&, double*, float*, float*, float*, PcgState*, double*,
                                          cudaStream_t);
template void cg_iteration<double, double>(const Op7<double>&, double*, double*, double*, double*, PcgState*,
                                           double*, cudaStream_t);
template void cg_iteration<float, float>(const Op7<float>&, float*, float*, float*, float*, PcgState*, double*,
                                         cudaStream_t);
template void cg_vector_updates<float, double>(const Op7<float>&, double*, float*, float*, float*, PcgState*, double*,
                                               cudaStream_t);

#define FS_KINST(V, RT)                                                                                           \
  template void pcg_init<V, RT>(const Op7<V>&, const RT*, RT*, RT*, V*, PcgState*, double*, cudaStream_t);       \
  template void pcg_resume<V, RT>(const Op7<V>&, const RT*, V*, PcgState*, double*, int, cudaStream_t);

FS_KINST(float, float)
FS_KINST(double, double)
FS_KINST(float, double)

}  // namespace fsb
