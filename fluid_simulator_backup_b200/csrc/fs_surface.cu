// The zero level set as a closed triangle mesh: the surface that
// WRITE_LEVELSET::WriteOBJ writes (WRITE_LEVELSET.h:22-84) through
// MARCHING_CUBES_ALGORITHM (MARCHING_CUBES_ALGORITHM.h:146-166, 497-757).
//
// The reference walks the cubes sequentially and shares each edge's vertex
// through pointer tables; here every stage is a data-parallel pass:
//   nodes      phi at the cube corners (the reference's trilinear sample)
//   cubes      inside/outside pattern per cube, -1 for a skipped cube, and
//              its triangle count
//   edges      one flag per grid edge that a kept cube crosses
//   scans      vertex numbers per flagged edge, triangle offsets per cube
//   vertices   the crossing on each flagged edge
//   triangles  per cube from the pattern's table, each turned along the
//              gradient of the cube's trilinear phi
//   normals    the normalised sum of the unit normals of a vertex's triangles
// Every stage uses correctly rounded operations without contraction, so the
// vertices and triangles are the bits of the CPU restatement of the same
// rules; vertex normals sum in fixed point, independent of the order.
//
// The triangle table is built here from the pattern, not copied: the surface
// crosses each face along segments between its sign-changing edges (a face
// with four crossings cuts off each inside corner, the same choice for the
// two cubes of the face, so the mesh is closed), the segments of the six
// faces close into loops, and each loop is fanned from its first edge.
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstring>

#include "fs_kernels.h"

namespace fsb {

namespace {

// corners: bit 0 the x offset, bit 1 y, bit 2 z; edges 0-3 along x, 4-7 y, 8-11 z
constexpr int kEdges[12][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3},
                               {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
constexpr int kFaces[6][4] = {{0, 2, 6, 4}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 3, 7, 6}, {0, 1, 3, 2}, {4, 5, 7, 6}};
constexpr int kMaxTri = 5;

struct McTable {
  signed char tri[256][3 * kMaxTri];
  int count[256];
};

__constant__ McTable c_table;

int edge_between(int a, int b) {
  for (int e = 0; e < 12; ++e)
    if ((kEdges[e][0] == a && kEdges[e][1] == b) || (kEdges[e][0] == b && kEdges[e][1] == a)) return e;
  return -1;
}

// Returns false if a pattern needed more than kMaxTri triangles.
bool build_table(McTable& t) {
  std::memset(&t, -1, sizeof t.tri);
  for (int mask = 0; mask < 256; ++mask) {
    int partner[12][2], np[12] = {0};
    for (const auto& f : kFaces) {
      int ring[4];
      bool in[4], act[4];
      int nact = 0;
      for (int q = 0; q < 4; ++q) {
        ring[q] = edge_between(f[q], f[(q + 1) % 4]);
        in[q] = (mask >> f[q]) & 1;
      }
      for (int q = 0; q < 4; ++q) {
        act[q] = in[q] != in[(q + 1) % 4];
        nact += act[q];
      }
      auto link = [&](int a, int b) {
        partner[a][np[a]++] = b;
        partner[b][np[b]++] = a;
      };
      if (nact == 2) {
        int s[2], m = 0;
        for (int q = 0; q < 4; ++q)
          if (act[q]) s[m++] = ring[q];
        link(s[0], s[1]);
      } else if (nact == 4) {
        for (int q = 0; q < 4; ++q)
          if (in[q]) link(ring[(q + 3) % 4], ring[q]);
      }
    }
    bool seen[12] = {false};
    int ntri = 0;
    for (int start = 0; start < 12; ++start) {
      if (np[start] == 0 || seen[start]) continue;
      int loop[12], len = 0, prev = -1, cur = start;
      seen[start] = true;
      loop[len++] = start;
      for (;;) {
        const int nxt = partner[cur][0] == prev ? partner[cur][1] : partner[cur][0];
        if (nxt == start) break;
        loop[len++] = nxt;
        seen[nxt] = true;
        prev = cur;
        cur = nxt;
      }
      for (int q = 1; q + 1 < len; ++q) {
        if (ntri == kMaxTri) return false;
        t.tri[mask][3 * ntri + 0] = (signed char)loop[0];
        t.tri[mask][3 * ntri + 1] = (signed char)loop[q];
        t.tri[mask][3 * ntri + 2] = (signed char)loop[q + 1];
        ++ntri;
      }
    }
    t.count[mask] = ntri;
  }
  return true;
}

// the low corner of edge e (kEdges[e][0]): x edges 0, 2, 4, 6; y edges 0, 1, 4, 5; z edges 0-3
__device__ __forceinline__ int edge_low_corner(int e) {
  return e < 4 ? 2 * e : (e < 8 ? ((e - 4) & 1) + 4 * ((e - 4) >> 1) : e - 8);
}

__device__ __forceinline__ double ra(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rs(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rm(double a, double b) { return __dmul_rn(a, b); }

// A cube corner's coordinate along one axis as the reference forms it
// (MARCHING_CUBES_ALGORITHM.h:151-166): centre of cube min(I, n-1) from the
// domain's low end, then -+ half a cell.
__device__ __forceinline__ double corner_coord(int I, int n, double dx) {
  const double half = rm(dx, 0.5);
  const int i = I < n - 1 ? I : n - 1;
  const double centre = ra(ra(0.0, half), rm(dx, (double)i));
  return I < n ? rs(centre, half) : ra(centre, half);
}

// Sample position -> clamped cell pair and weight along one axis
// (FIELD_STRUCTURE_3D.h:230-239; copied ghosts read as the clamped cells).
__device__ __forceinline__ void tri_axis(double pos, int n, double dx, double inv, int& i0, int& i1, double& a) {
  const int f = (int)floor(rs(rm(rs(pos, 0.0), inv), 0.5));
  a = rm(rs(pos, ra(0.0, rm(ra(0.5, (double)f), dx))), inv);
  i0 = f < 0 ? 0 : (f > n - 1 ? n - 1 : f);
  i1 = f + 1 < 0 ? 0 : (f + 1 > n - 1 ? n - 1 : f + 1);
}

struct NodeGrid {
  int nx, ny, nz;  // cells; nodes are (nx+1)(ny+1)(nz+1)
  __device__ __forceinline__ int64_t node(int I, int J, int K) const {
    return ((int64_t)K * (ny + 1) + J) * (nx + 1) + I;
  }
  __device__ __forceinline__ int64_t cube(int i, int j, int k) const { return ((int64_t)k * ny + j) * nx + i; }
  // edges of axis 0: [nz+1][ny+1][nx], 1: [nz+1][ny][nx+1], 2: [nz][ny+1][nx+1], concatenated
  __device__ __forceinline__ int64_t nxe() const { return (int64_t)(nz + 1) * (ny + 1) * nx; }
  __device__ __forceinline__ int64_t nye() const { return (int64_t)(nz + 1) * ny * (nx + 1); }
  __device__ __forceinline__ int64_t edge(int axis, int i, int j, int k) const {
    if (axis == 0) return ((int64_t)k * (ny + 1) + j) * nx + i;
    if (axis == 1) return nxe() + ((int64_t)k * ny + j) * (nx + 1) + i;
    return nxe() + nye() + ((int64_t)k * (ny + 1) + j) * (nx + 1) + i;
  }
};

template <class T>
__global__ void k_mc_nodes(const T* __restrict__ phi, Lay L, NodeGrid G, double dx, double* __restrict__ node) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  const int J = blockIdx.y * blockDim.y + threadIdx.y;
  const int K = blockIdx.z;
  if (I > G.nx || J > G.ny || K > G.nz) return;
  const double inv = 1.0 / dx;
  int i0, i1, j0, j1, k0, k1;
  double a, b, c;
  tri_axis(corner_coord(I, G.nx, dx), G.nx, dx, inv, i0, i1, a);
  tri_axis(corner_coord(J, G.ny, dx), G.ny, dx, inv, j0, j1, b);
  tri_axis(corner_coord(K, G.nz, dx), G.nz, dx, inv, k0, k1, c);
  const double v000 = (double)phi[L.at(i0, j0, k0)], v100 = (double)phi[L.at(i1, j0, k0)];
  const double v010 = (double)phi[L.at(i0, j1, k0)], v001 = (double)phi[L.at(i0, j0, k1)];
  const double v110 = (double)phi[L.at(i1, j1, k0)], v101 = (double)phi[L.at(i1, j0, k1)];
  const double v011 = (double)phi[L.at(i0, j1, k1)], v111 = (double)phi[L.at(i1, j1, k1)];
  const double ma = rs(1.0, a), mb = rs(1.0, b), mc = rs(1.0, c);
  const double mamb = rm(ma, mb), bc = rm(b, c);
  double v = rm(v000, rm(mamb, mc));
  v = ra(v, rm(rm(rm(a, mb), mc), v100));
  v = ra(v, rm(rm(rm(ma, b), mc), v010));
  v = ra(v, rm(rm(mamb, c), v001));
  v = ra(v, rm(rm(rm(a, b), mc), v110));
  v = ra(v, rm(rm(rm(a, mb), c), v101));
  v = ra(v, rm(rm(ma, bc), v011));
  v = ra(v, rm(rm(a, bc), v111));
  node[G.node(I, J, K)] = v == 0.0 ? -1e-8 : v;  // MARCHING_CUBES_ALGORITHM.h:308
}

// Pattern per cube (-1: skipped, a corner at 4 dx or more,
// MARCHING_CUBES_ALGORITHM.h:310-316) and its triangle count.
__global__ void k_mc_cubes(const double* __restrict__ node, NodeGrid G, double big, int* __restrict__ pattern,
                           int* __restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= G.nx || j >= G.ny || k >= G.nz) return;
  int mask = 0;
  bool kept = true;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const double v = node[G.node(i + (q & 1), j + (q >> 1 & 1), k + (q >> 2 & 1))];
    kept = kept && v < big;
    if (v <= 0.0) mask |= 1 << q;
  }
  const int64_t c = G.cube(i, j, k);
  pattern[c] = kept ? mask : -1;
  count[c] = kept ? c_table.count[mask] : 0;
}

// One flag per edge of the given axis: the sign changes along it and a kept
// cube has it.
__global__ void k_mc_edges(const double* __restrict__ node, const int* __restrict__ pattern, NodeGrid G, int axis,
                           int* __restrict__ used) {
  const int ex = G.nx + (axis != 0), ey = G.ny + (axis != 1), ez = G.nz + (axis != 2);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= ex || j >= ey || k >= ez) return;
  const double p0 = node[G.node(i, j, k)];
  const double p1 = node[G.node(i + (axis == 0), j + (axis == 1), k + (axis == 2))];
  bool any = false;
  if ((p0 <= 0.0) != (p1 <= 0.0)) {
    // the up to four cubes around the edge: offsets -1/0 in the two other axes
    for (int s = 0; s < 4; ++s) {
      int ci = i, cj = j, ck = k;
      const int d0 = -(s & 1), d1 = -(s >> 1 & 1);
      if (axis == 0) { cj += d0; ck += d1; }
      else if (axis == 1) { ci += d0; ck += d1; }
      else { ci += d0; cj += d1; }
      if (ci < 0 || cj < 0 || ck < 0 || ci >= G.nx || cj >= G.ny || ck >= G.nz) continue;
      any = any || pattern[G.cube(ci, cj, ck)] >= 0;
    }
  }
  used[G.edge(axis, i, j, k)] = any ? 1 : 0;
}

// The crossing on each flagged edge: (|phi1| P0 + |phi0| P1) * (1/(|phi0| + |phi1|))
// (MARCHING_CUBES_ALGORITHM.h:346, VECTOR_3D.h:130-135).
__global__ void k_mc_vertices(const double* __restrict__ node, const int* __restrict__ used,
                              const int* __restrict__ vid, NodeGrid G, int axis, double dx, double* __restrict__ xyz) {
  const int ex = G.nx + (axis != 0), ey = G.ny + (axis != 1), ez = G.nz + (axis != 2);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= ex || j >= ey || k >= ez) return;
  const int64_t e = G.edge(axis, i, j, k);
  if (!used[e]) return;
  const int i1 = i + (axis == 0), j1 = j + (axis == 1), k1 = k + (axis == 2);
  const double p0 = node[G.node(i, j, k)], p1 = node[G.node(i1, j1, k1)];
  const double a0 = p0 > 0.0 ? p0 : -p0, a1 = p1 > 0.0 ? p1 : -p1;
  const double inv = __ddiv_rn(1.0, ra(a0, a1));
  const double P0[3] = {corner_coord(i, G.nx, dx), corner_coord(j, G.ny, dx), corner_coord(k, G.nz, dx)};
  const double P1[3] = {corner_coord(i1, G.nx, dx), corner_coord(j1, G.ny, dx), corner_coord(k1, G.nz, dx)};
  double* out = xyz + 3 * (int64_t)vid[e];
#pragma unroll
  for (int q = 0; q < 3; ++q) out[q] = rm(ra(rm(a1, P0[q]), rm(a0, P1[q])), inv);
}

__device__ __forceinline__ void cross_rn(const double* p0, const double* p1, const double* p2, double* n) {
  const double u0 = rs(p1[0], p0[0]), u1 = rs(p1[1], p0[1]), u2 = rs(p1[2], p0[2]);
  const double w0 = rs(p2[0], p0[0]), w1 = rs(p2[1], p0[1]), w2 = rs(p2[2], p0[2]);
  n[0] = rs(rm(u1, w2), rm(u2, w1));
  n[1] = rs(rm(u2, w0), rm(u0, w2));
  n[2] = rs(rm(u0, w1), rm(u1, w0));
}

// Triangles per cube from the table, each turned so that its normal
// (v1 - v0) x (v2 - v0) does not point against the gradient of the cube's
// trilinear phi at its centre (the reference turns them along the level
// set's interpolated normal, TRIANGLE::CorrectCCW, TRIANGULAR_SURFACE.cpp:539-561).
__global__ void k_mc_triangles(const double* __restrict__ node, const int* __restrict__ pattern,
                               const int* __restrict__ toff, const int* __restrict__ vid,
                               const double* __restrict__ xyz, NodeGrid G, int* __restrict__ tri) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= G.nx || j >= G.ny || k >= G.nz) return;
  const int64_t cb = G.cube(i, j, k);
  const int mask = pattern[cb];
  if (mask < 0 || c_table.count[mask] == 0) return;
  double c[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) c[q] = node[G.node(i + (q & 1), j + (q >> 1 & 1), k + (q >> 2 & 1))];
  const double g0 = rs(ra(ra(c[1], c[3]), ra(c[5], c[7])), ra(ra(c[0], c[2]), ra(c[4], c[6])));
  const double g1 = rs(ra(ra(c[2], c[3]), ra(c[6], c[7])), ra(ra(c[0], c[1]), ra(c[4], c[5])));
  const double g2 = rs(ra(ra(c[4], c[5]), ra(c[6], c[7])), ra(ra(c[0], c[1]), ra(c[2], c[3])));
  int* out = tri + 3 * (int64_t)toff[cb];
  for (int t = 0; t < c_table.count[mask]; ++t) {
    int v[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int e = c_table.tri[mask][3 * t + q];
      const int a = edge_low_corner(e);
      const int axis = e < 4 ? 0 : (e < 8 ? 1 : 2);
      v[q] = vid[G.edge(axis, i + (a & 1), j + (a >> 1 & 1), k + (a >> 2 & 1))];
    }
    double n[3];
    cross_rn(xyz + 3 * (int64_t)v[0], xyz + 3 * (int64_t)v[1], xyz + 3 * (int64_t)v[2], n);
    if (ra(ra(rm(n[0], g0), rm(n[1], g1)), rm(n[2], g2)) < 0.0) {
      const int s = v[1];
      v[1] = v[2];
      v[2] = s;
    }
    out[3 * t + 0] = v[0] + 1;  // OBJ numbering
    out[3 * t + 1] = v[1] + 1;
    out[3 * t + 2] = v[2] + 1;
  }
}

// VERTEX::DetermineNormal (TRIANGULAR_SURFACE.cpp:99-121): the unit normals
// of a vertex's triangles, summed, then normalised.  The sums are taken in
// 2^-40 fixed point with 64-bit integer atomics: integer addition does not
// depend on the order the triangles arrive in, so the normals (and the OBJ
// text) are the same from run to run; the quantisation is below 1e-12.
constexpr double kNormalScale = 1099511627776.0;  // 2^40
__global__ void k_mc_face_normals(const int* __restrict__ tri, int64_t nt, const double* __restrict__ xyz,
                                  unsigned long long* __restrict__ acc) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int a = tri[3 * t] - 1, b = tri[3 * t + 1] - 1, c = tri[3 * t + 2] - 1;
  double n[3];
  cross_rn(xyz + 3 * (int64_t)a, xyz + 3 * (int64_t)b, xyz + 3 * (int64_t)c, n);
  const double len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  if (!(len > 0.0)) return;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    // two's complement: adding the unsigned image of a negative count subtracts it
    const unsigned long long u = (unsigned long long)__double2ll_rn(n[q] / len * kNormalScale);
    atomicAdd(acc + 3 * (int64_t)a + q, u);
    atomicAdd(acc + 3 * (int64_t)b + q, u);
    atomicAdd(acc + 3 * (int64_t)c + q, u);
  }
}

__global__ void k_mc_normalize(const unsigned long long* __restrict__ acc, double* __restrict__ nrm, int64_t nv) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  double n[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) n[q] = (double)(long long)acc[3 * v + q] / kNormalScale;
  const double len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
#pragma unroll
  for (int q = 0; q < 3; ++q) nrm[3 * v + q] = len > 0.0 ? n[q] / len : 0.0;
}

// __constant__ memory belongs to the device context: the table is copied to
// the current device on every polygonisation (a few kB, next to the passes
// over the grid), so a context that was reset and rebuilt since the last
// call gets it again.  The host copy is built once.
cudaError_t ensure_table() {
  static McTable host_table;
  static bool built = build_table(host_table);
  if (!built) return cudaErrorInvalidValue;
  return cudaMemcpyToSymbol(c_table, &host_table, sizeof host_table);
}

// exclusive prefix sum of n ints into out; returns the total in *total
cudaError_t exclusive_scan(const int* in, int* out, int64_t n, int* total, cudaStream_t s) {
  size_t bytes = 0;
  cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, (int)n, s);
  if (e != cudaSuccess) return e;
  void* tmp = nullptr;
  if ((e = cudaMalloc(&tmp, bytes)) != cudaSuccess) return e;
  e = cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, (int)n, s);
  int last_in = 0, last_out = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&last_in, in + n - 1, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&last_out, out + n - 1, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(tmp);
  *total = last_in + last_out;
  return e;
}

}  // namespace

template <class T>
cudaError_t polygonize(const T* phi, const Lay& L, double dx, SurfaceMesh* mesh, cudaStream_t s) {
  cudaError_t e = ensure_table();
  if (e != cudaSuccess) return e;
  NodeGrid G{L.nx, L.ny, L.nz};
  const int64_t nnode = (int64_t)(L.nx + 1) * (L.ny + 1) * (L.nz + 1);
  const int64_t ncube = (int64_t)L.nx * L.ny * L.nz;
  const int64_t nedge = (int64_t)(L.nz + 1) * (L.ny + 1) * L.nx + (int64_t)(L.nz + 1) * L.ny * (L.nx + 1) +
                        (int64_t)L.nz * (L.ny + 1) * (L.nx + 1);
  if (nedge > 0x7fffffff) return cudaErrorInvalidValue;  // 32-bit scans and vertex numbers
  double* node = nullptr;
  int *pattern = nullptr, *count = nullptr, *toff = nullptr, *used = nullptr, *vid = nullptr;
  unsigned long long* nacc = nullptr;
  auto cleanup = [&] {
    cudaFree(node);
    cudaFree(pattern);
    cudaFree(count);
    cudaFree(toff);
    cudaFree(used);
    cudaFree(vid);
    cudaFree(nacc);
  };
#define MC_TRY(x)             \
  do {                        \
    e = (x);                  \
    if (e != cudaSuccess) {   \
      cleanup();              \
      return e;               \
    }                         \
  } while (0)
  MC_TRY(cudaMalloc(&node, nnode * sizeof(double)));
  MC_TRY(cudaMalloc(&pattern, ncube * sizeof(int)));
  MC_TRY(cudaMalloc(&count, ncube * sizeof(int)));
  MC_TRY(cudaMalloc(&toff, ncube * sizeof(int)));
  MC_TRY(cudaMalloc(&used, nedge * sizeof(int)));
  MC_TRY(cudaMalloc(&vid, nedge * sizeof(int)));
  const dim3 b(32, 8, 1);
  k_mc_nodes<T><<<dim3((L.nx + 1 + 31) / 32, (L.ny + 1 + 7) / 8, L.nz + 1), b, 0, s>>>(phi, L, G, dx, node);
  k_mc_cubes<<<dim3((L.nx + 31) / 32, (L.ny + 7) / 8, L.nz), b, 0, s>>>(node, G, 4.0 * dx, pattern, count);
  for (int axis = 0; axis < 3; ++axis) {
    const int ex = L.nx + (axis != 0), ey = L.ny + (axis != 1), ez = L.nz + (axis != 2);
    k_mc_edges<<<dim3((ex + 31) / 32, (ey + 7) / 8, ez), b, 0, s>>>(node, pattern, G, axis, used);
  }
  MC_TRY(cudaGetLastError());
  int nv = 0, nt = 0;
  MC_TRY(exclusive_scan(used, vid, nedge, &nv, s));
  MC_TRY(exclusive_scan(count, toff, ncube, &nt, s));
  mesh->release();
  MC_TRY(cudaMalloc(&mesh->xyz, std::max<int64_t>(nv, 1) * 3 * sizeof(double)));
  MC_TRY(cudaMalloc(&mesh->normals, std::max<int64_t>(nv, 1) * 3 * sizeof(double)));
  MC_TRY(cudaMalloc(&mesh->tri, std::max<int64_t>(nt, 1) * 3 * sizeof(int)));
  mesh->nv = nv;
  mesh->nt = nt;
  for (int axis = 0; axis < 3; ++axis) {
    const int ex = L.nx + (axis != 0), ey = L.ny + (axis != 1), ez = L.nz + (axis != 2);
    k_mc_vertices<<<dim3((ex + 31) / 32, (ey + 7) / 8, ez), b, 0, s>>>(node, used, vid, G, axis, dx, mesh->xyz);
  }
  k_mc_triangles<<<dim3((L.nx + 31) / 32, (L.ny + 7) / 8, L.nz), b, 0, s>>>(node, pattern, toff, vid, mesh->xyz, G,
                                                                          mesh->tri);
  MC_TRY(cudaMalloc(&nacc, std::max<int64_t>(nv, 1) * 3 * sizeof(unsigned long long)));
  MC_TRY(cudaMemsetAsync(nacc, 0, std::max<int64_t>(nv, 1) * 3 * sizeof(unsigned long long), s));
  if (nt > 0) k_mc_face_normals<<<(int)((nt + 255) / 256), 256, 0, s>>>(mesh->tri, nt, mesh->xyz, nacc);
  if (nv > 0) k_mc_normalize<<<(int)((nv + 255) / 256), 256, 0, s>>>(nacc, mesh->normals, nv);
  MC_TRY(cudaGetLastError());
  MC_TRY(cudaStreamSynchronize(s));
  cleanup();
#undef MC_TRY
  return cudaSuccess;
}

void SurfaceMesh::release() {
  cudaFree(xyz);
  cudaFree(normals);
  cudaFree(tri);
  xyz = normals = nullptr;
  tri = nullptr;
  nv = nt = 0;
}

template cudaError_t polygonize<float>(const float*, const Lay&, double, SurfaceMesh*, cudaStream_t);
template cudaError_t polygonize<double>(const double*, const Lay&, double, SurfaceMesh*, cudaStream_t);

}  // namespace fsb
