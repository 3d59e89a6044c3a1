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
// Kernels of one iteration:
//   k_rb_spmv_pipe  q = S p, p.q and alpha: the operands staged plane by plane
//                   in shared memory by cp.async a few planes ahead, tau of
//                   the red cells computed there into a ring of planes
//                   (couplings 12 B, black p 2 B, black q 2 B per cell, plus
//                   the tile halo)
//   k_cg_update / k_cg_pupdate (fs_krylov.cu) on the packed black vectors
//                   (7 + 15 B per cell: FP32 r, p, q, FP64 iterate, bf16 1/diag)
// = 38 bytes per cell and iteration, at half the iterations of the full
// Jacobi-PCG's 64.
#include <cuda_bf16.h>

#include <algorithm>

#include "fs_kernels.h"

namespace fsb {

Lay make_half_lay(const Lay& L) { return make_lay((L.nx + 1) / 2, L.ny, L.nz); }

namespace {

// ---------------------------------------------------------------------------
// q = S p, pipelined.  The same two stages and arithmetic as above, with every
// operand staged in shared memory: a block owns a tile of TX x TY packed
// slots (2 TX x TY cells) and walks a chunk of z planes; for each plane it
// copies, 16 bytes per cp.async, the plane's p (tile + 2-slot halo in y,
// 4 in x) and its three coupling arrays (tile + halo) into one stage of a
// ring of NS stages, DIST planes ahead of the plane being computed.  The
// copies of plane k+2+DIST are in flight while tau of plane k+1 and q of
// plane k are computed from the stages of planes k-1 .. k+2, so the kernel
// waits on memory once per chunk instead of once per plane.  HBM carries
// about 21 bytes per cell (the 16 of the operands plus the halo).
// ---------------------------------------------------------------------------
namespace rbp {
constexpr int TX = 32, TY = 8;              // tile of packed slots (threads)
constexpr int PW = TX + 8, PR = TY + 4;     // p stage: slots h0-4 .. h0+TX+3, rows j0-2 .. j0+TY+1
constexpr int CW = 2 * TX + 8;              // coupling stages: cells 2h0-4 .. 2h0+2TX+3
constexpr int XR = TY + 2, YR = TY + 3, ZR = TY + 2;  // rows j0-1 .. j0+TY (ax, az), .. j0+TY+1 (ay)
constexpr int OFF_X = PR * PW, OFF_Y = OFF_X + XR * CW, OFF_Z = OFF_Y + YR * CW, STAGE = OFF_Z + ZR * CW;
constexpr int CP = PR * (PW / 4), CX = XR * (CW / 4), CY = YR * (CW / 4), CZ = ZR * (CW / 4);
constexpr int CHUNKS = CP + CX + CY + CZ;   // 16-byte copies per plane
constexpr int TW = TX + 2, TH = TY + 2;     // tau plane: tile + one-slot halo
// DIST planes in flight beyond the four in use; NS = 4 + DIST stages
constexpr size_t smem_bytes(int dist) { return (size_t)(4 + dist) * STAGE * sizeof(float); }
static_assert(STAGE % 4 == 0 && OFF_X % 4 == 0 && OFF_Y % 4 == 0 && OFF_Z % 4 == 0, "16-byte aligned stage parts");
}  // namespace rbp

// Source of 16-byte copy t of the stage of plane kk and its offset in the
// stage (floats); nullptr when the four values lie outside the padded array
// (the stage gets zeros there, values no computation reads).
__host__ __device__ inline const float* rb_chunk_src(const RbOp& A, const float* p, int h0, int j0, int kk, int t,
                                                     int* dst) {
  using namespace rbp;
  const float* base;
  const Lay* Y;
  int w, off, row0, col0;
  if (t < CP) {
    base = p; Y = &A.Lh; w = PW; off = 0; row0 = j0 - 2; col0 = h0 - 4;
  } else if ((t -= CP) < CX) {
    base = A.ax; Y = &A.L; w = CW; off = OFF_X; row0 = j0 - 1; col0 = 2 * h0 - 4;
  } else if ((t -= CX) < CY) {
    base = A.ay; Y = &A.L; w = CW; off = OFF_Y; row0 = j0 - 1; col0 = 2 * h0 - 4;
  } else {
    t -= CY;
    base = A.az; Y = &A.L; w = CW; off = OFF_Z; row0 = j0 - 1; col0 = 2 * h0 - 4;
  }
  const int r = t / (w / 4), c4 = t % (w / 4);
  *dst = off + r * w + 4 * c4;
  const int j = row0 + r;
  const int col = col0 + GX + 4 * c4;  // column within the padded row (a multiple of 4)
  if (j + GH < 0 || j + GH >= Y->py || kk + GH < 0 || kk + GH >= Y->nz + 2 * GH || col < 0 || col + 3 >= Y->px)
    return nullptr;
  return base + ((int64_t)(kk + GH) * Y->py + (j + GH)) * Y->px + col;
}

// Operand access in a stage (tile origin h0, j0).
__host__ __device__ inline int rb_sp(int h0, int j0, int h, int j) {
  return (j - (j0 - 2)) * rbp::PW + (h - (h0 - 4));
}
__host__ __device__ inline int rb_sc(int h0, int j0, int i, int j) {
  return (j - (j0 - 1)) * rbp::CW + (i - (2 * h0 - 4));
}

// tau of the red cell in slot (h, j, k) from the stages of planes k-1, k, k+1
// (the expression of rb_tau_at, operand for operand).
__host__ __device__ inline float rb_tau_s(const RbOp& A, const float* sm, const float* s0, const float* sp, int h0,
                                          int j0, int h, int j, int k, float e0) {
  using namespace rbp;
  const Lay& L = A.L;
  const Lay& H = A.Lh;
  if (h < 0 || j < 0 || k < 0 || h >= H.nx || j >= H.ny || k >= H.nz) return 0.0f;
  const int pr = (j + k) & 1;
  const int i = 2 * h + pr;
  if (i >= L.nx) return 0.0f;
  const float pxm = s0[rb_sp(h0, j0, h + pr - 1, j)], pxp = s0[rb_sp(h0, j0, h + pr, j)];
  const float pym = s0[rb_sp(h0, j0, h, j - 1)], pyp = s0[rb_sp(h0, j0, h, j + 1)];
  const float pzm = sm[rb_sp(h0, j0, h, j)], pzp = sp[rb_sp(h0, j0, h, j)];
  const float axm = s0[OFF_X + rb_sc(h0, j0, i, j)], axp = s0[OFF_X + rb_sc(h0, j0, i + 1, j)];
  const float aym = s0[OFF_Y + rb_sc(h0, j0, i, j)], ayp = s0[OFF_Y + rb_sc(h0, j0, i, j + 1)];
  const float azm = s0[OFF_Z + rb_sc(h0, j0, i, j)], azp = sp[OFF_Z + rb_sc(h0, j0, i, j)];
  const float b0 = i > 0 ? pxm : pxp;
  float num = axm * (pxm - b0) + axp * (pxp - b0);
  num += aym * (pym - b0) + ayp * (pyp - b0);
  num += azm * (pzm - b0) + azp * (pzp - b0);
  float d = ((axm + axp) + (aym + ayp)) + (azm + azp);
  if (i == 0 && j == 0 && k == 0) {
    num -= e0 * b0;
    d += e0;
  }
  return d > 0.0f ? num / d : 0.0f;
}

// (S p) of the black cell in slot (h, j, k), in-tile slot (tx, ty), from the
// stages of planes k-1, k, k+1 and the tau planes k-1, k, k+1 (tile + halo).
__host__ __device__ inline float rb_q_s(const RbOp& A, const float* sm, const float* s0, const float* sp,
                                        const float* tm, const float* t0, const float* tp, int h0, int j0, int h, int j,
                                        int k, float* pc_out) {
  using namespace rbp;
  const int pb = (j + k + 1) & 1;
  const int i = 2 * h + pb;
  *pc_out = 0.0f;
  if (i >= A.L.nx) return 0.0f;
  const int tx = h - h0 + 1, ty = j - j0 + 1;
  const float pc = s0[rb_sp(h0, j0, h, j)];
  const float axm = s0[OFF_X + rb_sc(h0, j0, i, j)], axp = s0[OFF_X + rb_sc(h0, j0, i + 1, j)];
  const float aym = s0[OFF_Y + rb_sc(h0, j0, i, j)], ayp = s0[OFF_Y + rb_sc(h0, j0, i, j + 1)];
  const float azm = s0[OFF_Z + rb_sc(h0, j0, i, j)], azp = sp[OFF_Z + rb_sc(h0, j0, i, j)];
  const float txm = t0[ty * TW + tx + pb - 1], txp = t0[ty * TW + tx + pb];
  const float tym = t0[(ty - 1) * TW + tx], typ = t0[(ty + 1) * TW + tx];
  const float tzm = tm[ty * TW + tx], tzp = tp[ty * TW + tx];
  const int o = i > 0 ? pb - 1 : 0;
  const float dxm = i > 1 ? pc - s0[rb_sp(h0, j0, h - 1, j)] : 0.0f;
  const float dym = pc - s0[rb_sp(h0, j0, h + o, j - 1)], dyp = pc - s0[rb_sp(h0, j0, h + o, j + 1)];
  const float dzm = pc - sm[rb_sp(h0, j0, h + o, j)], dzp = pc - sp[rb_sp(h0, j0, h + o, j)];
  float acc = axm * (dxm - txm) + axp * (0.0f - txp);
  acc += aym * (dym - tym) + ayp * (dyp - typ);
  acc += azm * (dzm - tzm) + azp * (dzp - tzp);
  *pc_out = pc;
  return acc;
}

namespace {

__device__ __forceinline__ void cp_async16(float* dst, const float* src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int DIST>
__global__ void __launch_bounds__(rbp::TX * rbp::TY) k_rb_spmv_pipe(RbOp A, const float* __restrict__ p,
                                                                    float* __restrict__ q, PcgState* st,
                                                                    double* partials, int kchunk) {
  using namespace rbp;
  constexpr int NS = 4 + DIST;
  if (((volatile PcgState*)st)->done) return;
  extern __shared__ float4 stage_mem[];
  float* stages = reinterpret_cast<float*>(stage_mem);
  __shared__ float ring[3 * TW * TH];
  const Lay& H = A.Lh;
  const int h0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int k0 = blockIdx.z * kchunk, k1 = min(H.nz, k0 + kchunk);
  const int tid = threadIdx.x + TX * threadIdx.y;
  const float e0 = (float)(*A.extra0);
  auto stage = [&](int kk) { return stages + ((kk % NS + NS) % NS) * STAGE; };
  auto load = [&](int kk) {
    if (kk <= k1 + 1) {
      float* d = stage(kk);
      for (int t = tid; t < CHUNKS; t += TX * TY) {
        int off;
        const float* s = rb_chunk_src(A, p, h0, j0, kk, t, &off);
        if (s)
          cp_async16(d + off, s);
        else
          *reinterpret_cast<float4*>(d + off) = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    cp_async_commit();  // one group per plane, empty past the chunk
  };
  auto tau_plane = [&](int kk) {
    float* dst = ring + ((kk % 3 + 3) % 3) * (TW * TH);
    const float *sm = stage(kk - 1), *s0 = stage(kk), *sp = stage(kk + 1);
    for (int t = tid; t < TW * TH; t += TX * TY) {
      const int x = t % TW, y = t / TW;
      dst[t] = rb_tau_s(A, sm, s0, sp, h0, j0, h0 - 1 + x, j0 - 1 + y, kk, e0);
    }
  };
  for (int kk = k0 - 2; kk <= k0 + 1 + DIST; ++kk) load(kk);
  cp_async_wait<DIST>();  // planes k0-2 .. k0+1 landed
  __syncthreads();
  tau_plane(k0 - 1);
  tau_plane(k0);
  const int h = h0 + threadIdx.x, j = j0 + threadIdx.y;
  const bool own = h < H.nx && j < H.ny;
  double pq = 0.0;
  for (int k = k0; k < k1; ++k) {
    cp_async_wait<DIST - 1>();  // plane k+2 landed
    __syncthreads();            // every thread is past plane k-1: its stage slot and tau slot are free
    load(k + 2 + DIST);
    tau_plane(k + 1);
    __syncthreads();
    if (own) {
      float pc;
      const float qv = rb_q_s(A, stage(k - 1), stage(k), stage(k + 1), ring + ((k + 2) % 3) * (TW * TH),
                              ring + (k % 3) * (TW * TH), ring + ((k + 1) % 3) * (TW * TH), h0, j0, h, j, k, &pc);
      q[H.at(h, j, k)] = qv;
      pq += (double)pc * (double)qv;
    }
  }
  pq = block_sum(pq);
  double tot;
  if (grid_reduce_sum(pq, partials, &st->ticket, &tot)) {
    st->pq = tot;
    const double alpha = st->rz / tot;
    if (!(tot > 0.0) || !isfinite(alpha)) {
      st->status = PCG_STAGNATED;
      st->done = 1;
      st->x_pending = 0;
    } else {
      st->alpha = alpha;
      st->x_pending = 1;
    }
  }
}

}  // namespace

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


// Launch shape of the pipelined SpMV: xy tiles times as many z chunks as
// fill one wave of resident blocks (a chunk costs 4 + DIST plane copies of
// prologue, so fewer and longer chunks are cheaper once the wave is full).
constexpr int kRbDist = 2;
struct RbLaunch {
  dim3 grid;
  int kchunk;
};
static int g_rb_resident = 0;  // resident blocks of the SpMV on this device (one wave)

void rb_prepare() {
  if (g_rb_resident > 0) return;
  cudaFuncSetAttribute(k_rb_spmv_pipe<kRbDist>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)rbp::smem_bytes(kRbDist));
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rb_spmv_pipe<kRbDist>, rbp::TX * rbp::TY,
                                                rbp::smem_bytes(kRbDist));
  g_rb_resident = std::max(1, per_sm) * std::max(1, sms);
}

RbLaunch rb_launch(const Lay& H) {
  const int tx = (H.nx + rbp::TX - 1) / rbp::TX, ty = (H.ny + rbp::TY - 1) / rbp::TY;
  const int resident = g_rb_resident > 0 ? g_rb_resident : 148;
  const int chunks = std::max(1, std::min(H.nz, resident / std::max(1, tx * ty)));
  const int kchunk = (H.nz + chunks - 1) / chunks;
  return {dim3(tx, ty, (H.nz + kchunk - 1) / kchunk), kchunk};
}

int rb_blocks(const Lay& H) {
  rb_prepare();
  const RbLaunch g = rb_launch(H);
  return std::max((int)(g.grid.x * g.grid.y * g.grid.z), reduction_blocks((int64_t)H.nx * H.ny * H.nz));
}

void rb_iteration(const RbOp& A, const Op7<float>& Ah, double* xh, float* rh, float* ph, float* qh, PcgState* st,
                  double* partials, cudaStream_t s) {
  const RbLaunch g = rb_launch(A.Lh);
  k_rb_spmv_pipe<kRbDist><<<g.grid, dim3(rbp::TX, rbp::TY, 1), rbp::smem_bytes(kRbDist), s>>>(A, ph, qh, st,
                                                                                              partials, g.kchunk);
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
