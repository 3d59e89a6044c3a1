// Red-black reduced pressure solve: the reference's PCG (PCG_METHOD.cpp:4-126)
// in multicolour ordering, for the FP32 + FP64 refinement projection.
//
// Colour the cells red (i+j+k even) and black (odd).  The seven-point
// pressure operator couples only cells of different colours, so in red-black
// order
//     A = [ D_R   -C ]      S = D_B - C^T D_R^-1 C
//         [ -C^T  D_B ]
// and the red block is diagonal: the red unknowns are eliminated exactly,
// x_R = D_R^-1 (b_R + C x_B), and CG with the black Jacobi preconditioner
// runs on the Schur complement S over the black cells only.  For an operator
// whose graph is two-coloured the Jacobi-preconditioned spectrum {1 +- l}
// becomes {1 - l^2}: the condition number drops by (1 + l_max)^2 -> 4 and
// CG needs half the iterations (714 -> 357 at 64^3 on the rising-bubble
// system), on vectors of half the length.
//
// Storage.  The black vectors (r, p, q, the FP64 iterate) and the red
// intermediate tau live in a packed half layout Lh: slot (h, j, k) holds the
// cell of its colour at i = 2h + parity, parity (j+k)&1 for red and
// (j+k+1)&1 for black, so each colour's row is contiguous and 16-byte
// aligned (float4 access in the vector kernels).  The couplings stay in the
// cell layout of the pressure operator (Op7: ax, ay, az, FP32).
//
// Applying S with FP32 accuracy.  S p = D_B p - C^T (D_R^-1 C p) cancels
// like diag*p - sum(a p): for the smooth error components its FP32 error
// would be eps32 * cond(A) relative.  Written per black cell c with the
// weighted average t_r = (sum_b a_rb p_b) / d_r of each red neighbour r,
//     (S p)_c = sum_r a_cr (p_c - t_r)           (d_c = sum_r a_cr),
// and t_r is carried as an offset from one of r's black neighbours b0(r):
//     tau_r = t_r - p_b0 = (sum_b a_rb (p_b - p_b0) - e_r p_b0) / d_r,
// d_r = sum_b a_rb + e_r (e_r: the deflation term of the first cell, 0
// elsewhere; d_r is summed from the same FP32 couplings, so the weights are
// the operator's own).  Every difference p_b - p_b0 and p_c - p_b0 is one
// of neighbouring values, correct to eps32 of itself, so (S p)_c =
// sum_r a_cr ((p_c - p_b0(r)) - tau_r) keeps the flux form's accuracy
// (eps32 of the fluxes, not of |p|).  b0(r) is r's x-1 neighbour, or its
// x+1 neighbour for r at i = 0.
//
// Kernels of one iteration (each array element once per kernel):
//   k_rb_red    tau of every red cell          reads ax, ay, az, p     writes tau
//   k_rb_black  q = S p                        reads ax, ay, az, p, tau writes q
//   k_pq_alpha  p.q and alpha                  reads p, q
//   k_cg_update / k_cg_pupdate (fs_krylov.cu) on the packed black vectors
// = 16 + 18 + 4 + 7 + 15 = 60 bytes per cell and iteration (FP32 couplings
// and vectors, FP64 black iterate, bf16 black pivots), at half the
// iterations of the full Jacobi-PCG's 64.
#include <cuda_bf16.h>

#include <algorithm>

#include "fs_kernels.h"

namespace fsb {

Lay make_half_lay(const Lay& L) { return make_lay((L.nx + 1) / 2, L.ny, L.nz); }

namespace {

// q = S p in two passes.  The red pass writes tau of every red cell, the
// black pass reads the couplings, p and the six tau of each black cell and
// writes q; each is one thread per packed slot and plane of a 4-plane z
// chunk, a (32, 8) tile of slots per block.  p.q and the step length follow
// in a separate streaming pass over p and q (pq_alpha, fs_krylov.cu).
// Both passes are plain streaming kernels with few instructions per cell:
// measured at 256^3 they run faster than fused forms that keep tau on chip
// (a z-marching shared-memory ring, and a cp.async-staged pipeline), whose
// per-plane barriers and index arithmetic made them issue- and
// latency-bound.
constexpr int kRbBY = 8;

// tau of the red cell in slot (h, j, k) (in range)
__device__ __forceinline__ float rb_tau(const RbOp& A, const float* __restrict__ p, int h, int j, int k) {
  const Lay& L = A.L;
  const Lay& H = A.Lh;
  const int pr = (j + k) & 1;
  const int i = 2 * h + pr;
  if (i >= L.nx) return 0.0f;
  const int64_t s = H.at(h, j, k);
  const int64_t c = L.at(i, j, k);
  // the six black neighbours (packed) and the couplings of the six faces
  const float pxm = p[s + pr - 1], pxp = p[s + pr];
  const float pym = p[s - H.px], pyp = p[s + H.px];
  const float pzm = p[s - H.slab], pzp = p[s + H.slab];
  const float axm = A.ax[c], axp = A.ax[c + 1];
  const float aym = A.ay[c], ayp = A.ay[c + L.px];
  const float azm = A.az[c], azp = A.az[c + L.slab];
  const float b0 = i > 0 ? pxm : pxp;
  float num = axm * (pxm - b0) + axp * (pxp - b0);
  num += aym * (pym - b0) + ayp * (pyp - b0);
  num += azm * (pzm - b0) + azp * (pzp - b0);
  float d = ((axm + axp) + (aym + ayp)) + (azm + azp);
  if (i == 0 && j == 0 && k == 0) {
    const float e0 = (float)(*A.extra0);
    num -= e0 * b0;
    d += e0;
  }
  return d > 0.0f ? num / d : 0.0f;
}

__global__ void __launch_bounds__(32 * kRbBY) k_rb_red(RbOp A, const float* __restrict__ p, float* __restrict__ tau,
                                                      const PcgState* st, int kchunk) {
  if (((volatile const PcgState*)st)->done) return;
  const int h = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * kRbBY + threadIdx.y;
  if (h >= A.Lh.nx || j >= A.Lh.ny) return;
  const int k0 = blockIdx.z * kchunk, k1 = min(A.Lh.nz, k0 + kchunk);
  for (int k = k0; k < k1; ++k) tau[A.Lh.at(h, j, k)] = rb_tau(A, p, h, j, k);
}

__global__ void __launch_bounds__(32 * kRbBY) k_rb_black(RbOp A, const float* __restrict__ p,
                                                        const float* __restrict__ tau, float* __restrict__ q,
                                                        const PcgState* st, int kchunk) {
  if (((volatile const PcgState*)st)->done) return;
  const Lay& L = A.L;
  const Lay& H = A.Lh;
  const int h = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * kRbBY + threadIdx.y;
  if (h < H.nx && j < H.ny) {
    const int k0 = blockIdx.z * kchunk, k1 = min(H.nz, k0 + kchunk);
    for (int k = k0; k < k1; ++k) {
      const int pb = (j + k + 1) & 1;
      const int i = 2 * h + pb;
      const int64_t s = H.at(h, j, k);
      float qv = 0.0f;
      if (i < L.nx) {
        const int64_t c = L.at(i, j, k);
        const float pc = p[s];
        const float axm = A.ax[c], axp = A.ax[c + 1];
        const float aym = A.ay[c], ayp = A.ay[c + L.px];
        const float azm = A.az[c], azp = A.az[c + L.slab];
        // tau of the six red neighbours
        const float txm = tau[s + pb - 1], txp = tau[s + pb];
        const float tym = tau[s - H.px], typ = tau[s + H.px];
        const float tzm = tau[s - H.slab], tzp = tau[s + H.slab];
        // b0 of each red neighbour: its x-1 black neighbour (x+1 at i = 0).
        // x-1 neighbour (at i-1): b0 is the black cell at i-2, or c itself when
        // i-1 = 0; x+1 neighbour: b0 is c.  y/z neighbours (at i): b0 is the
        // black cell at i-1 of their row (slot h + pb - 1), or at i+1 = 1
        // (slot 0) when i = 0.
        const int o = i > 0 ? pb - 1 : 0;
        const float dxm = i > 1 ? pc - p[s - 1] : 0.0f;
        const float dym = pc - p[s - H.px + o], dyp = pc - p[s + H.px + o];
        const float dzm = pc - p[s - H.slab + o], dzp = pc - p[s + H.slab + o];
        float acc = axm * (dxm - txm) + axp * (0.0f - txp);
        acc += aym * (dym - tym) + ayp * (dyp - typ);
        acc += azm * (dzm - tzm) + azp * (dzp - tzp);
        qv = acc;
      }
      q[s] = qv;
    }
  }
}

// The FP64 pressure from the packed black iterate: black cells copied, red
// cells eliminated exactly with the FP64 operator evaluated from phi (the
// same face coefficients and deflation term as the defect residual), so
// that the red rows of b - A p vanish to FP64 rounding:
// inv_dx2 (den p_c - sum_nb beta p_nb) = b_c  =>  p_c = (dx^2 b_c + sum) / den.
template <class T>
__global__ void k_rb_commit(const T* __restrict__ phi, const double* __restrict__ xh, const double* __restrict__ b,
                            double* __restrict__ p64, Lay L, Lay H, double rn, double rp, double dx2, int deflate) {
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (h >= H.nx || j >= H.ny || k >= H.nz) return;
  const int64_t s = H.at(h, j, k);
  const int pr = (j + k) & 1;
  const int ib = 2 * h + (1 - pr), ir = 2 * h + pr;
  if (ib < L.nx) p64[L.at(ib, j, k)] = xh[s];
  if (ir >= L.nx) return;
  const int64_t c = L.at(ir, j, k);
  const double pc = (double)phi[c];
  const double vneg = 1.0 / rn, vpos = 1.0 / rp;
  const int64_t nbc[6] = {c - 1, c + 1, c - L.px, c + L.px, c - L.slab, c + L.slab};
  const int64_t nbs[6] = {s + pr - 1, s + pr, s - H.px, s + H.px, s - H.slab, s + H.slab};
  const bool ok[6] = {ir > 0, ir < L.nx - 1, j > 0, j < L.ny - 1, k > 0, k < L.nz - 1};
  double sum = 0.0, den = 0.0;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    if (!ok[q]) continue;
    const double beta = face_coef(pc, (double)phi[nbc[q]], vneg, vpos);
    sum += beta * xh[nbs[q]];
    den += beta;
  }
  if (deflate && ir == 0 && j == 0 && k == 0) {
    // deflation: the betas of the bottom and down Neumann ghosts (POISSON_SOLVER_3D.h:1145-1179)
    const double vc = pc <= 0.0 ? vneg : vpos, acv = fabs(pc);
    const double gb = fabs(2.0 * pc - (double)phi[c + L.px]);
    const double gd = fabs(2.0 * pc - (double)phi[c + L.slab]);
    den += vc * vc * (gb + acv) / (vc * gb + vc * acv) + vc * vc * (gd + acv) / (vc * gd + vc * acv);
  }
  p64[c] = den > 0.0 ? (dx2 * b[c] + sum) / den : 0.0;
}

// packed black slots <- the black cells of a cell-layout field (FP64 iterate,
// FP32 residual, bf16 inverse diagonal); slots without a black cell get 0
template <class S, class D>
__global__ void k_rb_gather(const S* __restrict__ full, D* __restrict__ half, Lay L, Lay H) {
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (h >= H.nx || j >= H.ny || k >= H.nz) return;
  const int ib = 2 * h + ((j + k + 1) & 1);
  half[H.at(h, j, k)] = ib < L.nx ? (D)full[L.at(ib, j, k)] : D(0);
}

// The black pivots of IC(0) in red-black order.  Ordered red first, the
// incomplete Cholesky factor of A keeps the red block's diagonal (no fill
// there) and drops only the fill inside the black block, so its black
// pivots are diag(S) = d_c - sum_r a_cr^2 / d_r and PCG on A with that
// factor is PCG on the Schur complement S with the Jacobi preconditioner
// 1/diag(S).  Each term a_cr^2 / d_r is subtracted as a_cr (d_r - a_cr)/d_r,
// with d_r - a_cr the sum of r's other couplings, so nothing cancels.
// Written as bf16 1/diag(S) per packed black slot (0 for slots without a
// cell).
__global__ void k_rb_schur_dinv(RbOp A, unsigned short* __restrict__ dinv) {
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const Lay& L = A.L;
  const Lay& H = A.Lh;
  if (h >= H.nx || j >= H.ny || k >= H.nz) return;
  const int i = 2 * h + ((j + k + 1) & 1);
  const int64_t s = H.at(h, j, k);
  if (i >= L.nx) {
    dinv[s] = 0;
    return;
  }
  const int64_t c = L.at(i, j, k);
  const int64_t nb[6] = {c - 1, c + 1, c - L.px, c + L.px, c - L.slab, c + L.slab};
  const double a[6] = {A.ax[c], A.ax[c + 1], A.ay[c], A.ay[c + L.px], A.az[c], A.az[c + L.slab]};
  const int64_t c0 = L.at(0, 0, 0);
  double piv = 0.0;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    if (!(a[q] > 0.0)) continue;  // wall faces carry no coupling
    const int64_t r = nb[q];
    const double ar[6] = {A.ax[r], A.ax[r + 1], A.ay[r], A.ay[r + L.px], A.az[r], A.az[r + L.slab]};
    double other = r == c0 ? (double)*A.extra0 : 0.0;  // the deflation term of the first cell
    double dr = other;
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      dr += ar[m];
      if (m != (q ^ 1)) other += ar[m];  // r's face toward c is the opposite side of c's face q
    }
    piv += a[q] * (other / dr);
  }
  dinv[s] = __bfloat16_as_ushort(__float2bfloat16_rn(piv > 0.0 ? (float)(1.0 / piv) : 1.0f));
}

dim3 rb_grid(const Lay& H) { return dim3((H.nx + 31) / 32, (H.ny + 3) / 4, (H.nz + 1) / 2); }
const dim3 kRbBlock(32, 4, 2);

}  // namespace


// Launch shapes: xy tiles times z chunks, kRbChunk planes per block in the
// black pass, kRbRedChunk in the red pass.  Measured at 256^3 (CUDA events,
// one kernel at a time): the red pass takes 94 us with one block per tile
// and plane, 59 us with 2 planes per block and 54 us with 4 (a thread per
// cell is bound by block scheduling: each block lives about as long as one
// round trip to memory); the black pass 98 us with one plane per block and
// 66-74 us with 4 to 32.  The black pass reducing p.q itself took 95-97 us.
constexpr int kRbChunk = 4;
constexpr int kRbRedChunk = 4;

dim3 rb_red_grid(const Lay& H) {
  return dim3((H.nx + 31) / 32, (H.ny + kRbBY - 1) / kRbBY, (H.nz + kRbRedChunk - 1) / kRbRedChunk);
}
dim3 rb_black_grid(const Lay& H) {
  return dim3((H.nx + 31) / 32, (H.ny + kRbBY - 1) / kRbBY, (H.nz + kRbChunk - 1) / kRbChunk);
}

int rb_blocks(const Lay& H) {
  const dim3 g = rb_black_grid(H);
  return std::max((int)(g.x * g.y * g.z), reduction_blocks((int64_t)H.nx * H.ny * H.nz));
}

void rb_iteration(const RbOp& A, const Op7<float>& Ah, double* xh, float* rh, float* ph, float* qh, float* tau,
                  PcgState* st, double* partials, cudaStream_t s) {
  k_rb_red<<<rb_red_grid(A.Lh), dim3(32, kRbBY, 1), 0, s>>>(A, ph, tau, st, kRbRedChunk);
  k_rb_black<<<rb_black_grid(A.Lh), dim3(32, kRbBY, 1), 0, s>>>(A, ph, tau, qh, st, kRbChunk);
  pq_alpha<float>(Ah, ph, qh, st, partials, s);
  cg_vector_updates<float, double>(Ah, xh, rh, ph, qh, st, partials, s);
}

template <class T>
void rb_commit(const T* phi, const double* xh, const double* b, double* p64, const Lay& L, const Lay& H, double dx,
               double rho_neg, double rho_pos, int deflate, cudaStream_t s) {
  k_rb_commit<T><<<rb_grid(H), kRbBlock, 0, s>>>(phi, xh, b, p64, L, H, rho_neg, rho_pos, dx * dx, deflate);
}

void rb_schur_dinv(const RbOp& A, unsigned short* dinv, cudaStream_t s) {
  k_rb_schur_dinv<<<rb_grid(A.Lh), kRbBlock, 0, s>>>(A, dinv);
}

template <class S, class D>
void rb_gather(const S* full, D* half, const Lay& L, const Lay& H, cudaStream_t s) {
  k_rb_gather<S, D><<<rb_grid(H), kRbBlock, 0, s>>>(full, half, L, H);
}

template void rb_commit<float>(const float*, const double*, const double*, double*, const Lay&, const Lay&, double,
                               double, double, int, cudaStream_t);
template void rb_commit<double>(const double*, const double*, const double*, double*, const Lay&, const Lay&, double,
                                double, double, int, cudaStream_t);
template void rb_gather<double, double>(const double*, double*, const Lay&, const Lay&, cudaStream_t);
template void rb_gather<float, float>(const float*, float*, const Lay&, const Lay&, cudaStream_t);
template void rb_gather<unsigned short, unsigned short>(const unsigned short*, unsigned short*, const Lay&,
                                                        const Lay&, cudaStream_t);

}  // namespace fsb
