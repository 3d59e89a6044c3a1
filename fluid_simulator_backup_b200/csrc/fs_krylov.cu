// Jacobi-preconditioned conjugate gradients on a matrix-free seven-point
// operator (PCG_METHOD.cpp:4-126 restated for the GPU).
//
// One iteration is three kernels:
//   spmv    q = A p and p.q                      (reads p, ax, ay, az, diag; writes q)
//   update  x += alpha p, r -= alpha q, r.z, r.r (reads x, p, r, q, diag; writes x, r)
//   pupdate p = r/diag + beta p                  (reads r, diag, p; writes p)
// z = r/diag is never stored.  Dot products are block-reduced in FP64 and
// finished by the last block of the grid (deterministic for a given launch
// shape), which also takes the scalar decisions (alpha, beta, convergence,
// iteration cap, NaN) and writes them to the PcgState in device memory.
// Every kernel starts by reading `done`, so batches of iterations captured
// in a CUDA graph cost a few microseconds per launch once converged.
#include "fs_kernels.h"

namespace fsb {

constexpr int KB_X = 32, KB_Y = 4, KB_Z = 2;  // 256 threads

int pcg_blocks(const Lay& L) {
  return ((L.nx + KB_X - 1) / KB_X) * ((L.ny + KB_Y - 1) / KB_Y) * ((L.nz + KB_Z - 1) / KB_Z);
}

static inline Launch3 kl(const Lay& L) { return launch3(L.nx, L.ny, L.nz, KB_X, KB_Y, KB_Z); }

template <class V>
__device__ __forceinline__ V apply7(const Op7<V>& A, const V* __restrict__ x, int64_t c) {
  const int64_t sx = 1, sy = A.L.px, sz = A.L.slab;
  V acc = A.diag[c] * x[c];
  acc -= A.ax[c] * x[c - sx] + A.ax[c + sx] * x[c + sx];
  acc -= A.ay[c] * x[c - sy] + A.ay[c + sy] * x[c + sy];
  acc -= A.az[c] * x[c - sz] + A.az[c + sz] * x[c + sz];
  return acc;
}

// Three FP64 sums through one grid reduction.
__device__ __forceinline__ bool grid_reduce3(double a, double b, double c, double* partials, unsigned int* ticket,
                                             double out[3]) {
  __shared__ bool is_last;
  __shared__ double tot[3];
  a = block_sum(a);
  __syncthreads();
  b = block_sum(b);
  __syncthreads();
  c = block_sum(c);
  const int nb = num_blocks();
  const int blk = flat_block();
  if (thread0()) {
    partials[blk] = a;
    partials[nb + blk] = b;
    partials[2 * nb + blk] = c;
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    is_last = (t == (unsigned int)(nb - 1));
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  for (int m = 0; m < 3; ++m) {
    double s = 0.0;
    for (int q = tid; q < nb; q += nt) s += ((volatile double*)partials)[m * nb + q];
    s = block_sum(s);
    if (tid == 0) tot[m] = s;
    __syncthreads();
  }
  if (tid == 0) {
    out[0] = tot[0];
    out[1] = tot[1];
    out[2] = tot[2];
    *ticket = 0u;
  }
  return tid == 0;
}

template <class V>
__global__ void __launch_bounds__(256) k_pcg_init(Op7<V> A, const V* __restrict__ b, V* __restrict__ x,
                                                  V* __restrict__ r, V* __restrict__ p, PcgState* st,
                                                  double* partials) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  double rz = 0.0, rr = 0.0, bb = 0.0;
  if (i < A.L.nx && j < A.L.ny && k < A.L.nz) {
    const int64_t c = A.L.at(i, j, k);
    const V rv = b[c] - apply7(A, x, c);
    const V z = rv / A.diag[c];
    r[c] = rv;
    p[c] = z;
    rz = (double)rv * (double)z;
    rr = (double)rv * (double)rv;
    bb = (double)b[c] * (double)b[c];
  }
  double tot[3];
  if (grid_reduce3(rz, rr, bb, partials, &st->ticket, tot)) {
    st->rz = tot[0];
    st->rr = tot[1];
    st->bb = tot[2];
    st->iter = 0;
    st->beta = 0.0;
    st->best_rr = tot[1];
    st->stall = 0;
    st->status = PCG_RUNNING;
    st->done = 0;
    const bool nonfinite = !isfinite(tot[0]) || !isfinite(tot[1]);
    const bool converged = st->criterion == 1 ? (tot[0] < st->tol * st->tol)
                                              : (sqrt(tot[1]) <= st->tol * sqrt(tot[2]));
    if (nonfinite) {
      st->status = PCG_NONFINITE;
      st->done = 1;
    } else if (tot[2] == 0.0 || tot[1] == 0.0 || (converged && st->criterion == 0)) {
      // zero right-hand side or an exact initial guess: nothing to do
      st->status = PCG_CONVERGED;
      st->done = 1;
    } else if (st->max_iter <= 0) {
      st->status = PCG_MAXITER;
      st->done = 1;
    }
  }
}

template <class V>
__global__ void __launch_bounds__(256) k_pcg_spmv(Op7<V> A, const V* __restrict__ p, V* __restrict__ q, PcgState* st,
                                                  double* partials) {
  if (((volatile PcgState*)st)->done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  double pq = 0.0;
  if (i < A.L.nx && j < A.L.ny && k < A.L.nz) {
    const int64_t c = A.L.at(i, j, k);
    const V qv = apply7(A, p, c);
    q[c] = qv;
    pq = (double)p[c] * (double)qv;
  }
  pq = block_sum(pq);
  double tot;
  if (grid_reduce_sum(pq, partials, &st->ticket, &tot)) st->pq = tot;
}

template <class V>
__global__ void __launch_bounds__(256) k_pcg_update(Op7<V> A, V* __restrict__ x, V* __restrict__ r,
                                                    const V* __restrict__ p, const V* __restrict__ q, PcgState* st,
                                                    double* partials) {
  if (((volatile PcgState*)st)->done) return;
  const double pq_all = ((volatile PcgState*)st)->pq;
  const double alpha = ((volatile PcgState*)st)->rz / pq_all;
  // a non-positive p.Ap (or an infinite step) means the iteration has lost
  // its footing in this arithmetic: keep the iterate, stop (uniform branch)
  const bool breakdown = !(pq_all > 0.0) || !isfinite(alpha);
  const V a = (V)alpha;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  double rz = 0.0, rr = 0.0;
  if (!breakdown && i < A.L.nx && j < A.L.ny && k < A.L.nz) {
    const int64_t c = A.L.at(i, j, k);
    x[c] += a * p[c];
    const V rv = r[c] - a * q[c];
    r[c] = rv;
    rz = (double)rv * (double)(rv / A.diag[c]);
    rr = (double)rv * (double)rv;
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
    const bool nonfinite = !isfinite(tot[0]) || !isfinite(tot[1]);
    const bool converged = st->criterion == 1 ? (tot[0] < st->tol * st->tol)
                                              : (sqrt(tot[1]) <= st->tol * sqrt(st->bb));
    st->rz = tot[0];
    if (tot[1] < 0.99 * st->best_rr) {
      st->best_rr = tot[1];
      st->stall = 0;
    } else {
      st->stall += 1;
    }
    if (nonfinite) {
      st->status = PCG_NONFINITE;
      st->done = 1;
    } else if (converged) {
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
      }
    }
  }
}

template <class V>
__global__ void __launch_bounds__(256) k_pcg_pupdate(Op7<V> A, const V* __restrict__ r, V* __restrict__ p,
                                                     PcgState* st) {
  if (((volatile PcgState*)st)->done) return;
  const V beta = (V)((volatile PcgState*)st)->beta;
  FS_IJK(A.L);
  const int64_t c = A.L.at(i, j, k);
  p[c] = p[c] * beta + r[c] / A.diag[c];
}

template <class V>
void pcg_init(const Op7<V>& A, const V* b, V* x, V* r, V* p, PcgState* st, double* partials, cudaStream_t s) {
  Launch3 g = kl(A.L);
  k_pcg_init<V><<<g.grid, g.block, 0, s>>>(A, b, x, r, p, st, partials);
}

template <class V>
void pcg_iteration(const Op7<V>& A, V* x, V* r, V* p, V* q, PcgState* st, double* partials, cudaStream_t s) {
  Launch3 g = kl(A.L);
  k_pcg_spmv<V><<<g.grid, g.block, 0, s>>>(A, p, q, st, partials);
  k_pcg_update<V><<<g.grid, g.block, 0, s>>>(A, x, r, p, q, st, partials);
  k_pcg_pupdate<V><<<g.grid, g.block, 0, s>>>(A, r, p, st);
}

template void pcg_init<float>(const Op7<float>&, const float*, float*, float*, float*, PcgState*, double*,
                              cudaStream_t);
template void pcg_init<double>(const Op7<double>&, const double*, double*, double*, double*, PcgState*, double*,
                               cudaStream_t);
template void pcg_iteration<float>(const Op7<float>&, float*, float*, float*, float*, PcgState*, double*,
                                   cudaStream_t);
template void pcg_iteration<double>(const Op7<double>&, double*, double*, double*, double*, PcgState*, double*,
                                    cudaStream_t);

}  // namespace fsb
