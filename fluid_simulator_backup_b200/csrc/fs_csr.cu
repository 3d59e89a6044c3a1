// LINEAR_SOLVER plugin: Jacobi-PCG on a caller-supplied CSR matrix
// (LINEAR_SOLVER.h:36 / PCG_METHOD.cpp:4-126), for callers that keep the
// reference's assembled system.  The matrix-free operators of the projection
// and viscosity do not go through here; this entry point is the drop-in for
// `poisson_solver_type = "CUDAPCG"`-style use and for parity checks against
// the reference's own CSR systems.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/fluid_b200.h"
#include "fs_kernels.h"

using namespace fsb;

namespace {

struct CsrState {
  double rz, pq, rr, bb, tol;
  int iter, max_iter, done, criterion, status;
  unsigned int ticket;
  int bad_index;  // set by k_csr_init when row_ptr or column_index point outside the matrix
};

// status values of CsrState (0: running)
enum { CSR_CONVERGED = 1, CSR_MAXITER = 2, CSR_NONFINITE = 3, CSR_BAD_INDEX = 4 };

// r = b - A x, p = z = r/diag and the three start sums.  Every index is
// checked before it is used: a row whose row_ptr range leaves [0, nnz] or
// whose column index leaves [0, n) reads nothing and flags bad_index, which
// ends the solve before any other kernel reads the matrix (row_ptr must hold
// n + 1 entries and values/column_index nnz entries).
__global__ void k_csr_init(int n, int nnz, const double* __restrict__ val, const int* __restrict__ col,
                           const int* __restrict__ rp, const double* __restrict__ b, const double* __restrict__ x,
                           double* __restrict__ r, double* __restrict__ p, double* __restrict__ dinv,
                           double* partials, CsrState* st) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  double rz = 0, rr = 0, bb = 0;
  if (row < n) {
    const int q0 = rp[row], q1 = rp[row + 1];
    bool ok = 0 <= q0 && q0 <= q1 && q1 <= nnz;
    double acc = 0.0, d = 0.0;
    for (int q = q0; ok && q < q1; ++q) {
      const int cq = col[q];
      if (cq < 0 || cq >= n) { ok = false; break; }
      acc += val[q] * x[cq];
      if (cq == row) d = val[q];
    }
    if (!ok) {
      atomicOr(&st->bad_index, 1);
      d = 1.0;
      acc = b[row];
    }
    const double rv = b[row] - acc;
    const double di = 1.0 / d;
    dinv[row] = di;
    r[row] = rv;
    p[row] = rv * di;
    rz = rv * rv * di;
    rr = rv * rv;
    bb = b[row] * b[row];
  }
  __shared__ double sh[3][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  rz = warp_sum(rz); rr = warp_sum(rr); bb = warp_sum(bb);
  if (lane == 0) { sh[0][wid] = rz; sh[1][wid] = rr; sh[2][wid] = bb; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, c = 0, e = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { a += sh[0][w]; c += sh[1][w]; e += sh[2][w]; }
    atomicAdd(&partials[0], a);
    atomicAdd(&partials[1], c);
    atomicAdd(&partials[2], e);
  }
}

__global__ void k_csr_spmv(int n, const double* __restrict__ val, const int* __restrict__ col,
                           const int* __restrict__ rp, const double* __restrict__ p, double* __restrict__ q,
                           double* partials, const CsrState* st) {
  if (((volatile const CsrState*)st)->done) return;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  double pq = 0;
  if (row < n) {
    double acc = 0.0;
    for (int k = rp[row]; k < rp[row + 1]; ++k) acc += val[k] * p[col[k]];
    q[row] = acc;
    pq = p[row] * acc;
  }
  pq = warp_sum(pq);
  if ((threadIdx.x & 31) == 0) atomicAdd(&partials[3], pq);
}

__global__ void k_csr_update(int n, double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                             const double* __restrict__ q, const double* __restrict__ dinv, double* partials,
                             const CsrState* st) {
  if (((volatile const CsrState*)st)->done) return;
  const double alpha = ((volatile const CsrState*)st)->rz / ((volatile double*)partials)[3];
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  double rz = 0, rr = 0;
  if (row < n) {
    x[row] += alpha * p[row];
    const double rv = r[row] - alpha * q[row];
    r[row] = rv;
    rz = rv * rv * dinv[row];
    rr = rv * rv;
  }
  rz = warp_sum(rz);
  rr = warp_sum(rr);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&partials[4], rz);
    atomicAdd(&partials[5], rr);
  }
}

// scalar decisions between the update and the direction update
__global__ void k_csr_decide(double* partials, CsrState* st) {
  if (st->done) return;
  const double rz_new = partials[4], rr = partials[5];
  const double alpha = st->rz / partials[3];
  const bool bad = !isfinite(rz_new) || !isfinite(rr) || !isfinite(alpha);
  const bool conv = st->criterion == 1 ? rz_new < st->tol * st->tol : sqrt(rr) <= st->tol * sqrt(st->bb);
  partials[6] = rz_new / st->rz;  // beta
  st->rz = rz_new;
  st->rr = rr;
  partials[3] = 0.0;
  partials[4] = 0.0;
  partials[5] = 0.0;
  if (bad) { st->status = CSR_NONFINITE; st->done = 1; return; }
  if (conv) { st->status = CSR_CONVERGED; st->done = 1; return; }
  st->iter += 1;
  if (st->iter >= st->max_iter) { st->status = CSR_MAXITER; st->done = 1; }
}

__global__ void k_csr_pupdate(int n, double* __restrict__ p, const double* __restrict__ r,
                              const double* __restrict__ dinv, const double* partials, const CsrState* st) {
  if (((volatile const CsrState*)st)->done) return;
  const double beta = ((volatile const double*)partials)[6];
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row < n) p[row] = p[row] * beta + r[row] * dinv[row];
}

// The start decisions.  Like PCG_METHOD::PCGMethod (PCG_METHOD.cpp:4-126,
// `while (num_iteration < max_iteration)`), a cap of 0 runs no iteration and
// leaves x as it came.
__global__ void k_csr_start(double* partials, CsrState* st) {
  st->rz = partials[0];
  st->rr = partials[1];
  st->bb = partials[2];
  st->iter = 0;
  st->done = 0;
  st->status = 0;
  partials[3] = partials[4] = partials[5] = partials[6] = 0.0;
  if (st->bad_index) { st->status = CSR_BAD_INDEX; st->done = 1; }
  else if (!isfinite(st->rz)) { st->status = CSR_NONFINITE; st->done = 1; }
  else if (st->bb == 0.0 || st->rr == 0.0) { st->status = CSR_CONVERGED; st->done = 1; }
  else if (st->criterion == 0 && sqrt(st->rr) <= st->tol * sqrt(st->bb)) { st->status = CSR_CONVERGED; st->done = 1; }
  else if (st->max_iter <= 0) { st->status = CSR_MAXITER; st->done = 1; }
}

}  // namespace

extern "C" fs_status fs_pcg_csr(fs_ctx* ctx, int n, int nnz, const double* values, const int* column_index,
                                const int* row_ptr, const double* b, double* x, double tolerance, int max_iteration,
                                int stop, int* iterations, double* residual) {
  (void)ctx;
  if (n <= 0 || nnz <= 0 || !values || !column_index || !row_ptr || !b || !x || max_iteration < 0 ||
      (stop != FS_STOP_RELATIVE && stop != FS_STOP_ABSOLUTE)) {
    return FS_INVALID_ARG;
  }
  if (row_ptr[0] != 0 || row_ptr[n] != nnz) return FS_INVALID_ARG;
  for (int r = 0; r < n; ++r) {
    if (row_ptr[r + 1] < row_ptr[r]) return FS_INVALID_ARG;
    bool has_diag = false;
    for (int q = row_ptr[r]; q < row_ptr[r + 1]; ++q) {
      if (column_index[q] < 0 || column_index[q] >= n) return FS_INVALID_ARG;
      if (column_index[q] == r && values[q] != 0.0) has_diag = true;
    }
    if (!has_diag) return FS_INVALID_ARG;  // Jacobi needs a nonzero diagonal
  }
  cudaStream_t s;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return FS_CUDA_ERROR;
  double *dval = nullptr, *db = nullptr, *dx = nullptr, *dr = nullptr, *dp = nullptr, *dq = nullptr, *dd = nullptr,
         *part = nullptr;
  int *dcol = nullptr, *drp = nullptr;
  CsrState* st = nullptr;
  CsrState host{};
  fs_status result = FS_OK;
  auto ok = [&](cudaError_t e) {
    if (e != cudaSuccess && result == FS_OK) result = (e == cudaErrorMemoryAllocation) ? FS_OOM : FS_CUDA_ERROR;
    return e == cudaSuccess;
  };
  const size_t nb = (size_t)n * sizeof(double);
  if (ok(cudaMalloc(&dval, (size_t)nnz * sizeof(double))) && ok(cudaMalloc(&dcol, (size_t)nnz * sizeof(int))) &&
      ok(cudaMalloc(&drp, (size_t)(n + 1) * sizeof(int))) && ok(cudaMalloc(&db, nb)) && ok(cudaMalloc(&dx, nb)) &&
      ok(cudaMalloc(&dr, nb)) && ok(cudaMalloc(&dp, nb)) && ok(cudaMalloc(&dq, nb)) && ok(cudaMalloc(&dd, nb)) &&
      ok(cudaMalloc(&part, 8 * sizeof(double))) && ok(cudaMalloc(&st, sizeof(CsrState)))) {
    host.tol = tolerance;
    host.max_iter = max_iteration;
    host.criterion = stop;
    ok(cudaMemcpyAsync(dval, values, (size_t)nnz * sizeof(double), cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(dcol, column_index, (size_t)nnz * sizeof(int), cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(drp, row_ptr, (size_t)(n + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(db, b, nb, cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(dx, x, nb, cudaMemcpyHostToDevice, s));
    ok(cudaMemsetAsync(part, 0, 8 * sizeof(double), s));
    ok(cudaMemcpyAsync(st, &host, sizeof(CsrState), cudaMemcpyHostToDevice, s));
    const int T = 256, B = (n + T - 1) / T;
    k_csr_init<<<B, T, 0, s>>>(n, nnz, dval, dcol, drp, db, dx, dr, dp, dd, part, st);
    k_csr_start<<<1, 1, 0, s>>>(part, st);
    const int batches = max_iteration / 16 + 2;
    for (int bt = 0; bt < batches && result == FS_OK; ++bt) {
      ok(cudaMemcpyAsync(&host, st, sizeof(CsrState), cudaMemcpyDeviceToHost, s));
      ok(cudaStreamSynchronize(s));
      if (host.done) break;
      for (int it = 0; it < 16; ++it) {
        k_csr_spmv<<<B, T, 0, s>>>(n, dval, dcol, drp, dp, dq, part, st);
        k_csr_update<<<B, T, 0, s>>>(n, dx, dr, dp, dq, dd, part, st);
        k_csr_decide<<<1, 1, 0, s>>>(part, st);
        k_csr_pupdate<<<B, T, 0, s>>>(n, dp, dr, dd, part, st);
      }
      ok(cudaGetLastError());
    }
    ok(cudaMemcpyAsync(&host, st, sizeof(CsrState), cudaMemcpyDeviceToHost, s));
    ok(cudaMemcpyAsync(x, dx, nb, cudaMemcpyDeviceToHost, s));
    ok(cudaStreamSynchronize(s));
  }
  cudaFree(dval); cudaFree(dcol); cudaFree(drp); cudaFree(db); cudaFree(dx); cudaFree(dr); cudaFree(dp);
  cudaFree(dq); cudaFree(dd); cudaFree(part); cudaFree(st);
  cudaStreamDestroy(s);
  if (result != FS_OK) return result;
  if (iterations) *iterations = host.iter;
  if (residual) *residual = stop == FS_STOP_ABSOLUTE ? std::sqrt(host.rz) : (host.bb > 0 ? std::sqrt(host.rr / host.bb) : 0.0);
  if (host.status == CSR_NONFINITE) return FS_NONFINITE;
  if (host.status == CSR_MAXITER) return FS_NOT_CONVERGED;
  return FS_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant.
//
// Some callers cannot allocate device memory when they solve: a host that
// owns a fixed device memory pool (an FFI/JNI embedding whose allocator is
// not ours), a real-time loop that must not take cudaMalloc's implicit
// device synchronisation, or code that runs the solve between other work it
// has already sized.  fs_pcg_csr_noalloc gives them the same Jacobi-PCG as
// fs_pcg_csr on matrices and vectors they already hold in device memory; its
// working vectors live in one file-scope __device__ array of fixed size
// (kNoAllocMaxRows rows, about 8.4 MB), held by every GPU that loads the
// library until the process exits.
// ---------------------------------------------------------------------------

namespace {

constexpr int kNoAllocMaxRows = 1 << 18;  // 262144 rows: a 64^3 pressure system

struct NoAllocScratch {
  double r[kNoAllocMaxRows];
  double p[kNoAllocMaxRows];
  double q[kNoAllocMaxRows];
  double dinv[kNoAllocMaxRows];
  double partials[8];
  CsrState st;
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Device address of the scratch array in the current device's context.  In
// host code the symbol is only a host-side stand-in, so the address is
// looked up with the caller's device current.  The lookup allocates nothing
// and is repeated on every call: a context that was reset and rebuilt since
// the last call (cudaDeviceReset in the embedding) may hold the array at
// another address.
fs_status noalloc_scratch(NoAllocScratch** out) {
  void* ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if (e != cudaSuccess || !ptr) return FS_CUDA_ERROR;
  *out = static_cast<NoAllocScratch*>(ptr);
  return FS_OK;
}

}  // namespace

extern "C" fs_status fs_pcg_csr_noalloc(int n, int nnz, const double* values, const int* column_index,
                                        const int* row_ptr, const double* b, double* x, double tolerance,
                                        int max_iteration, int stop, void* stream, int* iterations,
                                        double* residual) {
  if (n <= 0 || nnz <= 0 || !values || !column_index || !row_ptr || !b || !x || max_iteration < 0 ||
      (stop != FS_STOP_RELATIVE && stop != FS_STOP_ABSOLUTE)) {
    return FS_INVALID_ARG;
  }
  if (n > kNoAllocMaxRows) return FS_INVALID_ARG;  // beyond the fixed scratch: use fs_pcg_csr
  // an error left behind by the caller's earlier, unrelated work is not this
  // solve's failure: clear it before the first launch is checked
  (void)cudaGetLastError();
  NoAllocScratch* sc = nullptr;
  fs_status st0 = noalloc_scratch(&sc);
  if (st0 != FS_OK) return st0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  CsrState host{};
  host.tol = tolerance;
  host.max_iter = max_iteration;
  host.criterion = stop;
  auto ok = [](cudaError_t e) { return e == cudaSuccess; };
  // the scratch keeps the previous call's contents: clear the accumulators
  // and the solver state (bad_index included) before the first kernel
  if (!ok(cudaMemsetAsync(sc->partials, 0, sizeof(sc->partials), s)) ||
      !ok(cudaMemcpyAsync(&sc->st, &host, sizeof(CsrState), cudaMemcpyHostToDevice, s))) {
    return FS_CUDA_ERROR;
  }
  const int T = 256, B = (n + T - 1) / T;
  k_csr_init<<<B, T, 0, s>>>(n, nnz, values, column_index, row_ptr, b, x, sc->r, sc->p, sc->dinv, sc->partials,
                             &sc->st);
  k_csr_start<<<1, 1, 0, s>>>(sc->partials, &sc->st);
  if (!ok(cudaGetLastError())) return FS_CUDA_ERROR;
  const int batches = max_iteration / 16 + 2;
  for (int bt = 0; bt < batches; ++bt) {
    if (!ok(cudaMemcpyAsync(&host, &sc->st, sizeof(CsrState), cudaMemcpyDeviceToHost, s)) ||
        !ok(cudaStreamSynchronize(s))) {
      return FS_CUDA_ERROR;
    }
    if (host.done) break;
    for (int it = 0; it < 16; ++it) {
      k_csr_spmv<<<B, T, 0, s>>>(n, values, column_index, row_ptr, sc->p, sc->q, sc->partials, &sc->st);
      k_csr_update<<<B, T, 0, s>>>(n, x, sc->r, sc->p, sc->q, sc->dinv, sc->partials, &sc->st);
      k_csr_decide<<<1, 1, 0, s>>>(sc->partials, &sc->st);
      k_csr_pupdate<<<B, T, 0, s>>>(n, sc->p, sc->r, sc->dinv, sc->partials, &sc->st);
    }
    if (!ok(cudaGetLastError())) return FS_CUDA_ERROR;
  }
  if (!ok(cudaMemcpyAsync(&host, &sc->st, sizeof(CsrState), cudaMemcpyDeviceToHost, s)) ||
      !ok(cudaStreamSynchronize(s))) {
    return FS_CUDA_ERROR;
  }
  if (iterations) *iterations = host.iter;
  if (residual) *residual = stop == FS_STOP_ABSOLUTE ? std::sqrt(host.rz) : (host.bb > 0 ? std::sqrt(host.rr / host.bb) : 0.0);
  if (host.status == CSR_BAD_INDEX) return FS_INVALID_ARG;
  if (host.status == CSR_NONFINITE) return FS_NONFINITE;
  if (host.status == CSR_MAXITER) return FS_NOT_CONVERGED;
  return FS_OK;
}
