// Fast sweeping reinitialisation (LEVELSET_3D.h:601-610, 734-918).
//
// One call of the reference is a set-up (cells farther than 20 dx from the
// interface and cells with a face neighbour of the other sign are fixed, the
// others reset to +-20 dx), one ghost fill (face ghosts copy the boundary
// cell) and two Gauss-Seidel sweeps whose traversal signs follow
// sweep_direction % 4.
//
// A Gauss-Seidel sweep over (k, j, i) in the signs (sz, sy, sx) updates a
// cell after its three upwind neighbours and before its three downwind ones.
// So do the diagonal hyperplanes of the sweep: cell (i', j', k') in sweep
// coordinates (i' = i for sx > 0, nx-1-i otherwise, ...) lies on
// s = i' + j' + k', its upwind neighbours on s-1 and its downwind ones on
// s+1.  Updating the cells of one hyperplane in parallel, hyperplane after
// hyperplane, therefore reads exactly the values the sequential sweep reads
// (Detrixhe, Gibou and Min, "A parallel fast sweeping method for the Eikonal
// equation", J. Comput. Phys. 237, 2013), and with the same correctly
// rounded operations, no contraction, it writes the same bits.
//
// The reference's INCREASING_SORT3 (MACROS.h:61-68) assigns a3 twice and
// leaves a2 untouched when c < b < a, so a2 keeps the value of the cell
// updated before in the sweep order.  That carried value has no parallel
// form: FS_FLAG_SORT_TYPO runs the sweeps sequentially in one thread
// (k_fs_sweep_serial), for parity with the reference's output; the default
// path sorts correctly (a2 = b).
#include <algorithm>

#include "fs_kernels.h"

namespace fsb {

// correctly rounded arithmetic without contraction
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rn_sqrt(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rn_sqrt(float a) { return __fsqrt_rn(a); }

template <class T>
struct SweepConst {
  T h, hh, hh2, third;
};

// One cell of LEVELSET_3D::Sweep (LEVELSET_3D.h:866-910) from its centre and
// six face neighbours.  a2 is the sort's middle value; with typo it is only
// written where the reference writes it, and *stale_read is set when the
// typo branch reads it before any cell of the sweep wrote it.
template <class T>
__device__ __forceinline__ T sweep_cell(T pc, T xm, T xp, T ym, T yp, T zm, T zp, const SweepConst<T>& K, T& a2,
                                        bool typo, bool& a2_set, int* stale_read) {
  T a, b, c;
  if (pc > T(0)) {
    a = xm > xp ? xp : xm;
    b = ym > yp ? yp : ym;
    c = zm > zp ? zp : zm;
  } else {
    a = xm > xp ? xm : xp;
    b = ym > yp ? ym : yp;
    c = zm > zp ? zm : zp;
  }
  T a1, a3;
  if (a <= b) {
    if (b <= c) { a1 = a; a2 = b; a3 = c; }
    else if (a <= c) { a1 = a; a2 = c; a3 = b; }
    else { a1 = c; a2 = a; a3 = b; }
    a2_set = true;
  } else if (a <= c) {
    a1 = b; a2 = a; a3 = c;
    a2_set = true;
  } else if (b <= c) {
    a1 = b; a2 = c; a3 = a;
    a2_set = true;
  } else {
    a1 = c;
    a3 = a;
    if (!typo) {
      a2 = b;
      a2_set = true;
    } else if (!a2_set) {
      *stale_read = 1;
    }
  }
  if (pc > T(0)) {
    T upd = rn_add(a1, K.h);
    if (upd > a2) {
      const T d = rn_sub(a1, a2);
      upd = rn_mul(T(0.5), rn_add(rn_add(a1, a2), rn_sqrt(rn_sub(K.hh2, rn_mul(d, d)))));
      if (upd > a3) {
        const T t = rn_add(rn_add(a1, a2), a3);
        const T q = rn_sub(rn_add(rn_add(rn_mul(a1, a1), rn_mul(a2, a2)), rn_mul(a3, a3)), K.hh);
        upd = rn_mul(K.third, rn_add(t, rn_sqrt(rn_sub(rn_mul(t, t), rn_mul(T(3), q)))));
      }
    }
    return upd > pc ? pc : upd;
  }
  T upd = rn_sub(a3, K.h);
  if (upd < a2) {
    const T d = rn_sub(a3, a2);
    upd = rn_mul(T(0.5), rn_sub(rn_add(a3, a2), rn_sqrt(rn_sub(K.hh2, rn_mul(d, d)))));
    if (upd < a1) {
      const T t = rn_add(rn_add(a1, a2), a3);
      const T q = rn_sub(rn_add(rn_add(rn_mul(a1, a1), rn_mul(a2, a2)), rn_mul(a3, a3)), K.hh);
      upd = rn_mul(K.third, rn_sub(t, rn_sqrt(rn_sub(rn_mul(t, t), rn_mul(T(3), q)))));
    }
  }
  return upd > pc ? upd : pc;
}

// The set-up of FastSweepingMethod (LEVELSET_3D.h:736-781).  The reference
// marks neighbours while it scans, but a marked neighbour always has a
// neighbour of the other sign itself, so the fixed set is: far cells, and
// cells with a face neighbour of the other sign (a wall's ghost copies the
// cell, so walls never count).  Out of place: in is not written.
template <class T>
__global__ void k_fs_prepare(const T* __restrict__ in, T* __restrict__ out, unsigned char* __restrict__ fixed, Lay L,
                             T nb) {
  FS_IJK(L);
  const int64_t c = L.at(i, j, k);
  const T pc = in[c];
  bool fix = (pc > T(0) ? pc : -pc) > nb;
  if (!fix) {
    const bool pos = pc > T(0);
    fix = (i + 1 < L.nx && (in[c + 1] > T(0)) != pos) || (i > 0 && (in[c - 1] > T(0)) != pos) ||
          (j + 1 < L.ny && (in[c + L.px] > T(0)) != pos) || (j > 0 && (in[c - L.px] > T(0)) != pos) ||
          (k + 1 < L.nz && (in[c + L.slab] > T(0)) != pos) || (k > 0 && (in[c - L.slab] > T(0)) != pos);
  }
  out[c] = fix ? pc : (pc > T(0) ? nb : -nb);
  fixed[c] = fix ? 1 : 0;
}

// Face ghosts (first layer) copy the boundary cell: FillGhostCellsFrom
// (FIELD_STRUCTURE_3D.h:663-780); the sweeps read no other ghost.
template <class T>
__global__ void k_fs_ghost_faces(T* __restrict__ f, Lay L) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y * blockDim.y + threadIdx.y;
  const int face = blockIdx.z;  // 0,1: x-, x+; 2,3: y-, y+; 4,5: z-, z+
  if (face < 2) {
    if (a >= L.ny || b >= L.nz) return;
    const int i = face == 0 ? 0 : L.nx - 1;
    const int64_t c = L.at(i, a, b);
    f[face == 0 ? c - 1 : c + 1] = f[c];
  } else if (face < 4) {
    if (a >= L.nx || b >= L.nz) return;
    const int j = face == 2 ? 0 : L.ny - 1;
    const int64_t c = L.at(a, j, b);
    f[face == 2 ? c - L.px : c + L.px] = f[c];
  } else {
    if (a >= L.nx || b >= L.ny) return;
    const int k = face == 4 ? 0 : L.nz - 1;
    const int64_t c = L.at(a, b, k);
    f[face == 4 ? c - L.slab : c + L.slab] = f[c];
  }
}

// The cells of hyperplane s of a sweep in signs (sx, sy, sz): one thread per
// (j', k'), i' = s - j' - k'.
template <class T>
__global__ void k_fs_plane(T* __restrict__ f, const unsigned char* __restrict__ fixed, Lay L, int s, int sx, int sy,
                           int sz, SweepConst<T> K) {
  const int jp = blockIdx.x * blockDim.x + threadIdx.x;
  const int kp = blockIdx.y * blockDim.y + threadIdx.y;
  if (jp >= L.ny || kp >= L.nz) return;
  const int ip = s - jp - kp;
  if (ip < 0 || ip >= L.nx) return;
  const int i = sx > 0 ? ip : L.nx - 1 - ip;
  const int j = sy > 0 ? jp : L.ny - 1 - jp;
  const int k = sz > 0 ? kp : L.nz - 1 - kp;
  const int64_t c = L.at(i, j, k);
  if (fixed[c]) return;
  T a2 = T(0);
  bool a2_set = false;
  int unused = 0;
  f[c] = sweep_cell(f[c], f[c - 1], f[c + 1], f[c - L.px], f[c + L.px], f[c - L.slab], f[c + L.slab], K, a2, false,
                    a2_set, &unused);
}

// The reference's sequential sweep with its sort as written: one thread,
// z outermost, x innermost, a2 carried from cell to cell.
template <class T>
__global__ void k_fs_sweep_serial(T* __restrict__ f, const unsigned char* __restrict__ fixed, Lay L, int sx, int sy,
                                  int sz, SweepConst<T> K, int* stale_read) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  T a2 = T(0);
  bool a2_set = false;
  for (int kp = 0; kp < L.nz; ++kp) {
    const int k = sz > 0 ? kp : L.nz - 1 - kp;
    for (int jp = 0; jp < L.ny; ++jp) {
      const int j = sy > 0 ? jp : L.ny - 1 - jp;
      for (int ip = 0; ip < L.nx; ++ip) {
        const int i = sx > 0 ? ip : L.nx - 1 - ip;
        const int64_t c = L.at(i, j, k);
        if (fixed[c]) continue;
        f[c] = sweep_cell(f[c], f[c - 1], f[c + 1], f[c - L.px], f[c + L.px], f[c - L.slab], f[c + L.slab], K, a2,
                          true, a2_set, stale_read);
      }
    }
  }
}

namespace {
// traversal signs (x, y, z) of the two sweeps of sweep_direction % 4 (LEVELSET_3D.h:789-818)
constexpr int kSweepSigns[4][2][3] = {{{1, 1, 1}, {-1, -1, -1}},
                                      {{-1, 1, -1}, {1, -1, 1}},
                                      {{1, -1, -1}, {-1, 1, 1}},
                                      {{-1, -1, 1}, {1, 1, -1}}};
}  // namespace

template <class T>
int fast_sweeping(const T* in, T* out, unsigned char* fixed, const Lay& L, double dx, int direction, int pairs,
                  int typo, int* stale_read, cudaStream_t s) {
  int launches = 0;
  const Launch3 g = launch3(L.nx, L.ny, L.nz);
  k_fs_prepare<T><<<g.grid, g.block, 0, s>>>(in, out, fixed, L, T(20.0 * dx));
  const int m = std::max(L.nx, std::max(L.ny, L.nz));
  const dim3 gb(16, 16, 1), gg((m + 15) / 16, (m + 15) / 16, 6);
  k_fs_ghost_faces<T><<<gg, gb, 0, s>>>(out, L);
  launches += 2;
  SweepConst<T> K;
  K.h = T(dx);
  K.hh = K.h * K.h;
  K.hh2 = K.hh * T(2);
  K.third = T(1) / T(3);
  const dim3 pb(32, 8, 1), pg((L.ny + 31) / 32, (L.nz + 7) / 8, 1);
  const int planes = L.nx + L.ny + L.nz - 2;
  for (int p = 0; p < pairs; ++p) {
    const int d = ((direction + p) % 4 + 4) % 4;
    for (int w = 0; w < 2; ++w) {
      const int* sg = kSweepSigns[d][w];
      if (typo) {
        k_fs_sweep_serial<T><<<1, 1, 0, s>>>(out, fixed, L, sg[0], sg[1], sg[2], K, stale_read);
        launches += 1;
      } else {
        for (int pl = 0; pl < planes; ++pl)
          k_fs_plane<T><<<pg, pb, 0, s>>>(out, fixed, L, pl, sg[0], sg[1], sg[2], K);
        launches += planes;
      }
    }
  }
  return launches;
}

template int fast_sweeping<float>(const float*, float*, unsigned char*, const Lay&, double, int, int, int, int*,
                                  cudaStream_t);
template int fast_sweeping<double>(const double*, double*, unsigned char*, const Lay&, double, int, int, int, int*,
                                   cudaStream_t);

}  // namespace fsb
