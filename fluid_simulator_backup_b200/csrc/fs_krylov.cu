// Jacobi-preconditioned conjugate gradients on a matrix-free seven-point
// operator (PCG_METHOD.cpp:4-126 restated for the GPU), with optional
// reliable updates for the mixed-precision pressure solve.
//
// Vector types: V for the operator, the search direction p and q = A p; R
// for the iterate x, the residual r and the right-hand side b.  V = R = double is
// the FP64 path, V = R = float the viscosity solves in FP32 storage, and
// V = float, R = double the mixed-precision pressure solve: the residual
// recurrences x += alpha p, r -= alpha q and all scalars stay in FP64
// while every operator application streams FP32 (88 bytes per unknown and
// iteration).  FP32 rounding of x, r or q would be amplified by ||A|| or
// by the transient growth of the CG residual; rounding of p only perturbs
// the search direction, and q is computed from the rounded p itself.
//
// One iteration is three kernels:
//   spmv    q = A p and p.q                      (reads p, ax, ay, az, diag; writes q)
//   update  x += alpha p, r -= alpha q, r.z, r.r (reads x, p, r, q, diag; writes x, r)
//   pupdate p = r/diag + beta p                  (reads r, diag, p; writes p)
// z = r/diag is never stored: 68 bytes per unknown and iteration in FP32,
// 136 in FP64.  The kernels run grid-stride over a grid of a few blocks per
// SM; dot products are reduced in FP64 per block and finished by the last
// block (deterministic for a given grid), which also takes the scalar
// decisions (alpha, beta, convergence, caps, breakdown) and writes them to
// the PcgState in device memory.  Every kernel starts by reading `done`, so
// iterations captured in a CUDA graph cost microseconds once a solve stops.
//
// Reliable updates (Clark et al., "Solving lattice QCD systems of equations
// using mixed precision solvers on GPUs", 2010): in the FP32 pressure solve
// the update kernel pauses the iteration (done = 2) whenever the recursive
// residual has dropped by `reliable_delta` since the last true residual; the
// host then folds x into the FP64 pressure, recomputes the true residual in
// FP64 and resumes the same Krylov iteration (pcg_resume) with that residual,
// keeping the search direction.  The FP32 iteration therefore converges like
// one long CG instead of a sequence of restarted ones.
#include <algorithm>
#include <cstdlib>

#include "fs_kernels.h"

namespace fsb {

static int g_sm_count = 0;
static int g_blocks_per_sm = 6;  // 6 x 256 threads: fully resident for kernels up to 40 registers

int reduction_blocks(int64_t n) {
  if (g_sm_count <= 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) g_sm_count = 148;
    if (const char* e = std::getenv("FS_BLOCKS_PER_SM")) {  // tuning knob for launch-shape sweeps
      const int v = std::atoi(e);
      if (v >= 1 && v <= 16) g_blocks_per_sm = v;
    }
  }
  const int64_t want = (n + kRedThreads - 1) / kRedThreads;
  const int64_t cap = (int64_t)g_blocks_per_sm * g_sm_count;
  return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

int pcg_blocks(const Lay& L) { return reduction_blocks((int64_t)L.nx * L.ny * L.nz); }

// (A x)_c evaluated in the type X of x (the operator's coefficients are
// converted): FP32 iterates get FP32 arithmetic, FP64 iterates FP64.
// The flux form is always evaluated in FP64 (loads in their storage type):
// for smooth x the six fluxes nearly cancel, and FP32 arithmetic would lose
// about log10(n) digits of q to that cancellation; FP64 arithmetic costs no
// memory traffic and the SpMV stays bandwidth bound.
template <class V, class X>
__device__ __forceinline__ X apply7(const Op7<V>& A, const X* __restrict__ x, int64_t c) {
  const int64_t sy = A.L.px, sz = A.L.slab;
  const X xc = x[c];
  if (A.flux_form) {
    const double d = (double)xc;
    double acc = (double)A.ax[c] * (d - (double)x[c - 1]) + (double)A.ax[c + 1] * (d - (double)x[c + 1]);
    acc += (double)A.ay[c] * (d - (double)x[c - sy]) + (double)A.ay[c + sy] * (d - (double)x[c + sy]);
    acc += (double)A.az[c] * (d - (double)x[c - sz]) + (double)A.az[c + sz] * (d - (double)x[c + sz]);
    if (c == A.L.at(0, 0, 0)) acc += (*A.extra0) * d;
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
    for (int q = threadIdx.x; q < nb; q += blockDim.x) s += ((volatile double*)partials)[m * nb + q];
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
    const RT z = rv / (RT)A.diag[c];
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

template <class V>
__global__ void __launch_bounds__(kRedThreads) k_pcg_spmv(Op7<V> A, const V* __restrict__ p, V* __restrict__ q,
                                                          PcgState* st, double* partials) {
  if (((volatile PcgState*)st)->done) return;
  double pq = 0.0;
  Cursor cur;
  for (cur.init(A.L); cur.valid(A.L); cur.next(A.L)) {
    const int64_t c = A.L.at(cur.i, cur.j, cur.k);
    const V qv = apply7<V, V>(A, p, c);
    q[c] = qv;
    pq += (double)p[c] * (double)qv;  // p.q of the stored (rounded) q, as the update uses it
  }
  pq = block_sum(pq);
  double tot;
  if (grid_reduce_sum(pq, partials, &st->ticket, &tot)) st->pq = tot;
}

template <class V, class RT, class Q = V>
__global__ void __launch_bounds__(kRedThreads) k_pcg_update(Op7<V> A, RT* __restrict__ x, RT* __restrict__ r,
                                                            const V* __restrict__ p, const Q* __restrict__ q,
                                                            PcgState* st, double* partials) {
  if (((volatile PcgState*)st)->done) return;
  const double pq_all = ((volatile PcgState*)st)->pq;
  const double alpha = ((volatile PcgState*)st)->rz / pq_all;
  // a non-positive p.Ap (or an infinite step) means the iteration has lost
  // its footing in this arithmetic: keep the iterate, stop (uniform branch)
  const bool breakdown = !(pq_all > 0.0) || !isfinite(alpha);
  const RT ar = (RT)alpha;
  double rz = 0.0, rr = 0.0;
  if (!breakdown) {
    Cursor cur;
    for (cur.init(A.L); cur.valid(A.L); cur.next(A.L)) {
      const int64_t c = A.L.at(cur.i, cur.j, cur.k);
      x[c] += ar * (RT)p[c];
      const RT rv = r[c] - ar * (RT)q[c];
      r[c] = rv;
      rz += (double)rv * (double)(rv / (RT)A.diag[c]);
      rr += (double)rv * (double)rv;
    }
  }
  double tot[3];
  if (grid_reduce3(rz, rr, 0.0, partials, &st->ticket, tot)) {
    if (breakdown) {
      st->status = PCG_STAGNATED;
      st->done = 1;
      return;
    }
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

template <class V, class RT>
__global__ void __launch_bounds__(kRedThreads) k_pcg_pupdate(Op7<V> A, const RT* __restrict__ r, V* __restrict__ p,
                                                             PcgState* st) {
  if (((volatile PcgState*)st)->done) return;
  const RT beta = (RT)((volatile PcgState*)st)->beta;
  Cursor cur;
  for (cur.init(A.L); cur.valid(A.L); cur.next(A.L)) {
    const int64_t c = A.L.at(cur.i, cur.j, cur.k);
    p[c] = (V)((RT)p[c] * beta + r[c] / (RT)A.diag[c]);
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
    rz += (double)rv * (double)(rv / (RT)A.diag[c]);
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
void pcg_iteration(const Op7<V>& A, RT* x, RT* r, V* p, V* q, PcgState* st, double* partials, cudaStream_t s) {
  const int nb = pcg_blocks(A.L);
  k_pcg_spmv<V><<<nb, kRedThreads, 0, s>>>(A, p, q, st, partials);
  k_pcg_update<V, RT><<<nb, kRedThreads, 0, s>>>(A, x, r, p, q, st, partials);
  k_pcg_pupdate<V, RT><<<nb, kRedThreads, 0, s>>>(A, r, p, st);
}

// Stored-coefficient variant of the mixed iteration: FP32 face couplings in
// flux form, evaluated in FP64, q in FP64.
template <class V>
__global__ void __launch_bounds__(kRedThreads) k_pcg_spmv_q64(Op7<V> A, const V* __restrict__ p, double* __restrict__ q,
                                                              PcgState* st, double* partials) {
  if (((volatile PcgState*)st)->done) return;
  const int64_t sy = A.L.px, sz = A.L.slab;
  double pq = 0.0;
  Cursor cur;
  for (cur.init(A.L); cur.valid(A.L); cur.next(A.L)) {
    const int64_t c = A.L.at(cur.i, cur.j, cur.k);
    const double d = (double)p[c];
    double acc = (double)A.ax[c] * (d - (double)p[c - 1]) + (double)A.ax[c + 1] * (d - (double)p[c + 1]);
    acc += (double)A.ay[c] * (d - (double)p[c - sy]) + (double)A.ay[c + sy] * (d - (double)p[c + sy]);
    acc += (double)A.az[c] * (d - (double)p[c - sz]) + (double)A.az[c + sz] * (d - (double)p[c + sz]);
    if (c == A.L.at(0, 0, 0)) acc += (*A.extra0) * d;
    q[c] = acc;
    pq += d * acc;
  }
  pq = block_sum(pq);
  double tot;
  if (grid_reduce_sum(pq, partials, &st->ticket, &tot)) st->pq = tot;
}

void pcg_iteration_stored32(const Op7<float>& A, double* x, double* r, float* p, double* q, PcgState* st,
                            double* partials, cudaStream_t s) {
  const int nb = pcg_blocks(A.L);
  k_pcg_spmv_q64<float><<<nb, kRedThreads, 0, s>>>(A, p, q, st, partials);
  k_pcg_update<float, double, double><<<nb, kRedThreads, 0, s>>>(A, x, r, p, q, st, partials);
  k_pcg_pupdate<float, double><<<nb, kRedThreads, 0, s>>>(A, r, p, st);
}

template <class V, class RT>
void pcg_resume(const Op7<V>& A, const RT* r, V* p, PcgState* st, double* partials, int restart, cudaStream_t s) {
  const int nb = pcg_blocks(A.L);
  k_pcg_resume<V, RT><<<nb, kRedThreads, 0, s>>>(A, r, st, partials, restart);
  k_pcg_pupdate<V, RT><<<nb, kRedThreads, 0, s>>>(A, r, p, st);
}

#define FS_KINST(V, RT)                                                                                           \
  template void pcg_init<V, RT>(const Op7<V>&, const RT*, RT*, RT*, V*, PcgState*, double*, cudaStream_t);       \
  template void pcg_iteration<V, RT>(const Op7<V>&, RT*, RT*, V*, V*, PcgState*, double*, cudaStream_t);        \
  template void pcg_resume<V, RT>(const Op7<V>&, const RT*, V*, PcgState*, double*, int, cudaStream_t);

FS_KINST(float, float)
FS_KINST(double, double)
FS_KINST(float, double)

}  // namespace fsb
