// Shared device-side definitions of the B200 solver: padded array layout,
// launch helpers and block reductions.
//
// HBM layout.  Every field is a padded 3-D array with a ghost ring of width 3
// on all six sides (the WENO5 stencil reach), x fastest.  Stencil kernels
// therefore never branch on the box boundary: ghost values are written by a
// ghost-fill kernel (level set: linear extrapolation) or are permanently zero
// (velocity ghosts, pressure-solve vector ghosts, coefficient faces on walls).
// In x the interior starts at column 4 (one unused column before the three
// ghosts) and the row pitch px is a multiple of 4, so every interior row
// starts on a 16-byte boundary for FP32 and a 32-byte boundary for FP64:
// the streaming kernels move x-aligned groups of four cells with vector
// loads and stores.
// The reference stores the same x-fastest order (ARRAY_3D.h:98) with ghost
// widths 2-3 per field (EULERIAN_FLUID_SOLVER_3D.h:405-431).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fsb {

constexpr int GH = 3;  // ghost width
constexpr int GX = 4;  // column of i = 0 within a row (ghosts at GX-3 .. GX-1)

struct Lay {
  int nx, ny, nz;   // interior extent
  int px, py;       // padded extent in x (a multiple of 4) and y
  int64_t slab;     // px*py
  int64_t total;    // px*py*(nz+2*GH)
  __host__ __device__ int64_t at(int i, int j, int k) const {
    return ((int64_t)(k + GH) * py + (j + GH)) * px + (i + GX);
  }
};

inline Lay make_lay(int nx, int ny, int nz) {
  Lay l;
  l.nx = nx; l.ny = ny; l.nz = nz;
  l.px = (nx + GX + GH + 3) / 4 * 4;
  l.py = ny + 2 * GH;
  l.slab = (int64_t)l.px * l.py;
  l.total = l.slab * (nz + 2 * GH);
  return l;
}

// Interior launch: one thread per (i, j, k), x fastest.
struct Launch3 {
  dim3 grid, block;
};

inline Launch3 launch3(int nx, int ny, int nz, int bx = 32, int by = 4, int bz = 2) {
  Launch3 L;
  L.block = dim3(bx, by, bz);
  L.grid = dim3((nx + bx - 1) / bx, (ny + by - 1) / by, (nz + bz - 1) / bz);
  return L;
}

#define FS_IJK(L)                                      \
  const int i = blockIdx.x * blockDim.x + threadIdx.x; \
  const int j = blockIdx.y * blockDim.y + threadIdx.y; \
  const int k = blockIdx.z * blockDim.z + threadIdx.z; \
  if (i >= (L).nx || j >= (L).ny || k >= (L).nz) return;

// Grid-stride traversal of the interior of a layout, x fastest, for the
// reduction kernels: they run on a grid of a few blocks per SM (set by
// reduction_blocks), so the per-block partial sums and the one atomic
// ticket per block stay few.  The cursor advances (i, j, k) by the grid
// stride with carries instead of dividing every linear index.
struct Cursor {
  int i, j, k, si, sj, sk;
  __device__ __forceinline__ void init(const Lay& L) {
    const int64_t start = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t row = start / L.nx;
    i = (int)(start % L.nx);
    j = (int)(row % L.ny);
    k = (int)(row / L.ny);
    const int64_t srow = stride / L.nx;
    si = (int)(stride % L.nx);
    sj = (int)(srow % L.ny);
    sk = (int)(srow / L.ny);
  }
  __device__ __forceinline__ bool valid(const Lay& L) const { return k < L.nz; }
  __device__ __forceinline__ void next(const Lay& L) {
    i += si;
    int c = i >= L.nx;
    i -= c ? L.nx : 0;
    j += sj + c;
    c = j >= L.ny;
    j -= c ? L.ny : 0;
    k += sk + c;
  }
};

// Blocks for a grid-stride reduction kernel of 256 threads over n items.
int reduction_blocks(int64_t n);
constexpr int kRedThreads = 256;

// Ghost-fluid face coefficient of the pressure operator between cells with
// level sets pc, pn (POISSON_SOLVER_3D.h:1080-1085): with b = 1/rho of each
// cell's phase, beta = b_c b_n (|phi_n| + |phi_c|) / (b_n |phi_c| + b_c |phi_n|),
// which is b itself when both cells are in the same phase (evaluated as b
// there: the reference's expression gives b up to rounding).
// (vneg, vpos are 1/rho of the two phases, precomputed by the caller.)
__device__ __forceinline__ double face_coef(double pc, double pn, double vneg, double vpos) {
  const bool nc = pc <= 0.0, nn = pn <= 0.0;
  const double vc = nc ? vneg : vpos;
  if (nc == nn) return vc;
  const double vn = nn ? vneg : vpos;
  const double ac = fabs(pc), an = fabs(pn);
  return vc * vn * (an + ac) / (vn * ac + vc * an);
}

// Block-wide sum of a double (any block size that is a multiple of 32, up
// to 1024).  Result valid in thread 0.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double part[32];
  const int lane = (threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z)) & 31;
  const int warp = (threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z)) >> 5;
  const int nwarps = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) part[warp] = v;
  __syncthreads();
  v = 0.0;
  if (warp == 0) {
    v = lane < nwarps ? part[lane] : 0.0;
    v = warp_sum(v);
  }
  return v;
}

__device__ __forceinline__ double block_max(double v) {
  __shared__ double partm[32];
  const int lane = (threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z)) & 31;
  const int warp = (threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z)) >> 5;
  const int nwarps = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) partm[warp] = v;
  __syncthreads();
  v = 0.0;
  if (warp == 0) {
    v = lane < nwarps ? partm[lane] : 0.0;
    v = warp_max(v);
  }
  return v;
}

__device__ __forceinline__ int flat_block() { return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z); }
__device__ __forceinline__ int num_blocks() { return gridDim.x * gridDim.y * gridDim.z; }
__device__ __forceinline__ bool thread0() { return threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0; }

// Deterministic grid-wide reduction: every block writes its partial, the last
// block to finish (counted with an atomic ticket) sums the partials in a
// fixed order and resets the ticket.  Returns true in the one thread that holds
// the final value in *out_total (thread 0 of the last block).
__device__ __forceinline__ bool grid_reduce_sum(double block_value, double* partials, unsigned int* ticket,
                                                double* out_total) {
  __shared__ bool is_last;
  const int b = flat_block();
  if (thread0()) {
    partials[b] = block_value;
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    is_last = (t == (unsigned int)(num_blocks() - 1));
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  double s = 0.0;
  // L2 loads (.cg: the partials of this launch, not stale L1 lines of an
  // earlier one), not volatile, so that the loop's loads are in flight
  // together; the additions keep their order, so the sum is deterministic
  const int nbk = num_blocks();
#pragma unroll 8
  for (int q = tid; q < nbk; q += nt) s += __ldcg(partials + q);
  s = block_sum(s);
  if (tid == 0) {
    *out_total = s;
    *ticket = 0u;
    return true;
  }
  return false;
}

}  // namespace fsb
