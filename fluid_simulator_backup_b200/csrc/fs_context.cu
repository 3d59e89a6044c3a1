// fs_ctx: device state of one simulation and the C ABI of include/fluid_b200.h.
//
// The host side here replaces the reference's thread-pool runtime
// (MULTITHREADING.h, one fork/join per frame plus a barrier after every grid
// loop) with one CUDA stream per context: every operator is a short sequence
// of kernel launches on that stream, and the Krylov loops run as captured
// CUDA graphs of 16 iterations whose kernels stop themselves once the solve
// has converged, with one host check of the solver state per graph launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "../../include/fluid_b200.h"
#include "fs_kernels.h"

using namespace fsb;

namespace {

thread_local char g_last_error[512] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof g_last_error, fmt, ap);
  va_end(ap);
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return FS_CUDA_ERROR;                                                               \
    }                                                                                     \
  } while (0)

#define CKS(...)                   \
  do {                             \
    fs_status s_ = (__VA_ARGS__);  \
    if (s_ != FS_OK) return s_;    \
  } while (0)

constexpr int kGraphIters = 16;

// A device buffer typed at run time (float or double storage).
struct Buf {
  void* p = nullptr;
  size_t bytes = 0;
};

}  // namespace

struct fs_ctx {
  fs_grid_desc grid{};
  fs_params prm{};
  bool fp32 = false;  // storage precision of the fields
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  Lay Lc{}, Lu{}, Lv{}, Lw{};

  std::vector<Buf> owned;
  int64_t bytes = 0;

  // fields (storage type S)
  void *phi = nullptr, *s1 = nullptr, *s2 = nullptr, *s3 = nullptr, *s4 = nullptr, *sgn = nullptr;
  void *u = nullptr, *v = nullptr, *w = nullptr;
  void *u0 = nullptr, *v0 = nullptr, *w0 = nullptr;
  void *ua = nullptr, *va = nullptr, *wa = nullptr;
  // pressure (FP64) and projection work
  double *p64 = nullptr, *b64 = nullptr, *div64 = nullptr, *p64bak = nullptr;
  double* kappa = nullptr;  // mean curvature (surface tension)
  unsigned char* fsfixed = nullptr;  // fast sweeping: cells the sweeps leave alone
  int* fsflag = nullptr;             // fast sweeping: the reference's sort read its uninitialised a2
  int sweep_direction = 0;           // LEVELSET_3D::sweep_direction
  SurfaceMesh mesh;                  // the last fs_surface
  // pressure PCG in the solve precision V (double for FP64, float for FP32_REFINE)
  void *pax = nullptr, *pay = nullptr, *paz = nullptr, *pdiag = nullptr;
  unsigned short* pdinv = nullptr;  // bf16 1/diag: the Jacobi preconditioner of the FP32 pressure solve
  // red-black reduced FP32 pressure solve (packed half layout Lh, fs_redblack.cu)
  Lay Lh{};
  double* rb_x = nullptr;          // black FP64 iterate
  float *rb_r = nullptr, *rb_p = nullptr, *rb_q = nullptr, *rb_tau = nullptr;
  unsigned short* rb_dinv = nullptr;  // black bf16 1/diag
  PipeGeom pipe{};  // the oil/water pipe's geometry (pipe.on = 0: the box)
  void* pgen[3] = {nullptr, nullptr, nullptr};  // pipe: masked periodic velocity copies
  void* pgx[3] = {nullptr, nullptr, nullptr};   // pipe: their ENO3-guarded copies along x
  void* pgz[3] = {nullptr, nullptr, nullptr};   // and along z
  void *px = nullptr, *pr = nullptr, *pp = nullptr, *pq = nullptr, *prhs = nullptr;
  // viscosity systems, one per component (storage type S)
  void* vs[3][9] = {};  // ax, ay, az, diag, rhs, x, r, p, q
  // reductions
  double* partials = nullptr;
  unsigned int* tickets = nullptr;  // [8]
  double* scalars = nullptr;        // [16]
  PcgState* st = nullptr;           // device
  PcgState* st_host = nullptr;      // pinned
  double* sc_host = nullptr;        // pinned [16]
  double* staging = nullptr;        // packed FP64 transfer buffer
  // captured solver graphs keyed by solve kind and the one operand whose
  // buffer rotates between calls (the level set); kernel arguments are
  // baked into a graph, so a different buffer needs its own graph
  std::map<std::pair<int, const void*>, cudaGraphExec_t> graphs;
  // accounting for fs_step_report
  int64_t launches = 0;
  float pcg_ms = 0.0f;
  int pcg_launched_iterations = 0;
  cudaEvent_t evp0 = nullptr, evp1 = nullptr;
  // adjoint state (bars FP64 in both precisions; allocated on first use)
  double* abar[4] = {};       // bars of phi, u, v, w (FS_FIELD_ADJ_*)
  double* awork_c[6] = {};    // cell work bars
  double* awork_f[4][3] = {}; // face work bar triples
  double* a_vlam[3] = {};     // viscosity: lambda per component
  double* a_vxb[3] = {};      // viscosity: x_bar per component
  double* a_rho = nullptr;    // device [4]: bars of rho_neg, rho_pos
  std::vector<void*> tape_cells, tape_faces;  // taped forward states (storage precision), allocated on demand
  std::vector<double*> tape_p;                // taped stage pressures (FP64)
  // FP64 operator and Krylov vectors of the adjoint solves: the forward's own
  // buffers in FP64 contexts; FP32 contexts solve the pressure adjoint with
  // the mixed solve and keep one FP64 viscosity system set shared by the
  // three components
  double *a_ax = nullptr, *a_ay = nullptr, *a_az = nullptr, *a_diag = nullptr;
  double *a_r = nullptr, *a_p = nullptr, *a_q = nullptr;
  double* a_vs[3][9] = {};
  // derived from fs_params by apply_params
  bool debug = false;           // params.verbose: solver progress on stderr
  double reliable_delta = 0.1;  // params.reliable_delta
  int flux32 = 2;               // params.flux_arithmetic (Op7::flux32)
  int lean = 1;                 // FP32 pressure solve preconditioned by the bf16 inverse diagonal (Op7::dinv16)
  bool red_black = false;       // FP32 pressure solve on the red-black Schur complement
  bool rb_ic0 = true;           // its preconditioner: 1/diag(S) (IC(0) in red-black order), else the black 1/diag
  int adj_unconverged = 0;      // adjoint solves of the current call that stopped before their tolerance
  double adj_worst_rel = 0.0;   // and the worst relative residual they reached
  char adj_note[128] = {0};     // the last of them: which solve, its status and iterations

  size_t S() const { return fp32 ? sizeof(float) : sizeof(double); }
};

namespace {

// Forward states kept for the adjoint of one step.  Each pointer is a
// padded field of the context's layouts in its storage precision; the
// pressures are FP64.
struct Tape {
  void* ls[4] = {};                   // level set: the three RK stage inputs and the advected phi
  void* vel[3][3][3] = {};            // [stage][0 input, 1 viscosity input, 2 projection input][component]
  double* p[3] = {};                  // pressure of each stage's projection
  std::vector<void*> re[3];           // [reinit block][pseudo-step]: input of each Sussman step
};

fs_status dalloc(fs_ctx* c, void** out, size_t bytes) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error("cudaMalloc of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    return FS_OOM;
  }
  e = cudaMemsetAsync(p, 0, bytes, c->stream);
  if (e != cudaSuccess) {
    cudaFree(p);
    set_error("cudaMemsetAsync failed: %s", cudaGetErrorString(e));
    return FS_CUDA_ERROR;
  }
  c->owned.push_back({p, bytes});
  c->bytes += (int64_t)bytes;
  *out = p;
  return FS_OK;
}

void release(fs_ctx* c) {
  if (!c) return;
  for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);
  c->graphs.clear();
  for (auto& b : c->owned) cudaFree(b.p);
  c->owned.clear();
  c->mesh.release();
  if (c->st_host) cudaFreeHost(c->st_host);
  if (c->sc_host) cudaFreeHost(c->sc_host);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->evp0) cudaEventDestroy(c->evp0);
  if (c->evp1) cudaEventDestroy(c->evp1);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
}

const Lay& lay_of(const fs_ctx* c, int field) {
  switch (field) {
    case FS_FIELD_U: case FS_FIELD_ADJ_U: return c->Lu;
    case FS_FIELD_V: case FS_FIELD_ADJ_V: return c->Lv;
    case FS_FIELD_W: case FS_FIELD_ADJ_W: return c->Lw;
    default: return c->Lc;
  }
}

bool is_adjoint_field(int field) { return field >= FS_FIELD_ADJ_PHI && field <= FS_FIELD_ADJ_W; }

fs_status check_params(const fs_params* p) {
  if (!p) { set_error("params is NULL"); return FS_INVALID_ARG; }
  if (!(p->rho_neg > 0) || !(p->rho_pos > 0)) { set_error("densities must be positive"); return FS_INVALID_ARG; }
  if (p->mu_neg < 0 || p->mu_pos < 0) { set_error("viscosities must be non-negative"); return FS_INVALID_ARG; }
  if (p->order < 1 || p->order > 3) { set_error("order must be 1, 2 or 3"); return FS_INVALID_ARG; }
  if (p->precision != FS_PRECISION_FP64 && p->precision != FS_PRECISION_FP32_REFINE) {
    set_error("unknown precision %d", p->precision);
    return FS_INVALID_ARG;
  }
  if (p->stop != FS_STOP_RELATIVE && p->stop != FS_STOP_ABSOLUTE) { set_error("unknown stop criterion"); return FS_INVALID_ARG; }
  if (!(p->velocity_epsilon >= 0) || !std::isfinite(p->velocity_epsilon)) {
    set_error("velocity_epsilon must be finite and >= 0");
    return FS_INVALID_ARG;
  }
  if (p->viscosity < 0 || p->viscosity > 2) {
    set_error("viscosity must be 0 (off), 1 (semi-implicit) or 2 (explicit)");
    return FS_INVALID_ARG;
  }
  if (p->velocity_scheme != FS_VELOCITY_WENO5 && p->velocity_scheme != FS_VELOCITY_ENO3) {
    set_error("unknown velocity scheme %d", p->velocity_scheme);
    return FS_INVALID_ARG;
  }
  if (!(p->surface_tension >= 0) || !std::isfinite(p->surface_tension)) {
    set_error("surface_tension must be finite and non-negative");
    return FS_INVALID_ARG;
  }
  if (!(p->tolerance >= 0) || p->max_iteration < 0 || p->reinit_iterations < 0 || p->reinit_scaling <= 0) {
    set_error("bad solver or reinitialisation settings");
    return FS_INVALID_ARG;
  }
  if (p->pressure_preconditioner < FS_PRECOND_DEFAULT || p->pressure_preconditioner > FS_PRECOND_RED_BLACK_JACOBI ||
      (p->pressure_preconditioner >= FS_PRECOND_JACOBI_BF16 && p->precision != FS_PRECISION_FP32_REFINE)) {
    set_error("unknown pressure preconditioner %d for this precision", p->pressure_preconditioner);
    return FS_INVALID_ARG;
  }
  if (p->pipe && (p->pressure_preconditioner == FS_PRECOND_RED_BLACK ||
                  p->pressure_preconditioner == FS_PRECOND_RED_BLACK_JACOBI)) {
    set_error("the pipe mode's pressure solve takes the Jacobi preconditioners only");
    return FS_INVALID_ARG;
  }
  if (!(p->reliable_delta >= 0.0 && p->reliable_delta < 1.0)) {
    set_error("reliable_delta must be in [0, 1)");
    return FS_INVALID_ARG;
  }
  if (p->host_loop != 0 && p->host_loop != 1) {
    set_error("host_loop must be 0 or 1");
    return FS_INVALID_ARG;
  }
  if (p->flux_arithmetic < 0 || p->flux_arithmetic > 2) {
    set_error("flux_arithmetic must be 0, 1 or 2");
    return FS_INVALID_ARG;
  }
  if (p->precision == FS_PRECISION_FP32_REFINE && (!(p->inner_tolerance > 0) || p->max_outer < 1)) {
    set_error("FP32_REFINE needs inner_tolerance > 0 and max_outer >= 1");
    return FS_INVALID_ARG;
  }
  return FS_OK;
}

// The solver settings of the context that follow from its parameters.
void apply_params(fs_ctx* c) {
  const fs_params& p = c->prm;
  c->debug = p.verbose != 0;
  c->reliable_delta = p.reliable_delta > 0.0 ? p.reliable_delta : 0.1;
  c->flux32 = p.flux_arithmetic;
  c->lean = p.pressure_preconditioner != FS_PRECOND_JACOBI;
  // FP32_REFINE: the default is red-black IC(0), which halves the
  // iterations of the Jacobi-PCG (FP64 keeps the reference's Jacobi); the
  // pipe mode's default is the bf16 Jacobi (its red cells would need the
  // pipe's Neumann cells in the FP64 elimination)
  c->red_black = c->fp32 && !p.pipe && (p.pressure_preconditioner == FS_PRECOND_DEFAULT ||
                              p.pressure_preconditioner == FS_PRECOND_RED_BLACK ||
                              p.pressure_preconditioner == FS_PRECOND_RED_BLACK_JACOBI);
  c->rb_ic0 = p.pressure_preconditioner != FS_PRECOND_RED_BLACK_JACOBI;
}

// The pressure system keeps the reference's deflation of the first cell only
// in the faithful projection.  The corrected projection solves the singular
// Neumann system as it is (consistent: b has zero mean), so that the
// corrected velocity's divergence is the solve's residual in every cell;
// with the deflation the first cell's divergence would carry the sum of the
// residual, e0 p0 = -sum(r).
int deflate(const fs_ctx* c) { return (c->prm.flags & FS_FLAG_FAITHFUL_PROJECTION) ? 1 : 0; }
// The pipe's geometry for the projection kernels (nullptr in the box) and the
// cell that carries the deflation (-1: cell (0,0,0) of the box).
const PipeGeom* pipe_of(const fs_ctx* c) { return c->pipe.on ? &c->pipe : nullptr; }
int64_t deflated_cell(const fs_ctx* c) { return c->pipe.on ? c->Lc.at(c->pipe.fi, c->pipe.fj, c->pipe.fk) : -1; }

// The oil/water vertical pipe: its grids as the reference computes them (cell
// spacing (max - min)/(n - 1); each face grid reaches half a cell further on
// its own axis, GRID_STRUCTURE_3D.h:91-137, EULERIAN_FLUID_SOLVER_3D.h:
// 405-427) and the checks the mode needs.
fs_status setup_pipe(fs_ctx* c) {
  const fs_params& p = c->prm;
  c->pipe = PipeGeom{};
  if (p.pipe == 0) return FS_OK;
  if (p.pipe != 1) { set_error("pipe must be 0 (the box) or 1 (a vertical pipe)"); return FS_INVALID_ARG; }
  const int n[3] = {c->grid.nx, c->grid.ny, c->grid.nz};
  double d[3];
  for (int a = 0; a < 3; ++a) {
    d[a] = (p.grid_max[a] - p.grid_min[a]) / (n[a] - 1);
    if (!(d[a] > 0) || !std::isfinite(d[a]) || std::fabs(d[a] - c->grid.dx) > 1e-9 * c->grid.dx) {
      set_error("pipe mode: (grid_max - grid_min)/(n - 1) must equal the grid's dx on every axis");
      return FS_INVALID_ARG;
    }
  }
  if (!(p.pipe_radius > 0) || !(p.pipe_R1 > 0) || !(p.pipe_V0 != 0) || !std::isfinite(p.pipe_V0) ||
      !std::isfinite(p.pipe_f) || !(p.pipe_eta > 0) || !(p.pipe_oil_density > 0) || !(p.pipe_We > 0) ||
      !std::isfinite(p.pipe_We)) {
    set_error("pipe mode: pipe_radius, pipe_R1, pipe_eta, pipe_oil_density, pipe_We must be positive, pipe_V0 "
              "non-zero");
    return FS_INVALID_ARG;
  }
  if (n[1] < 5) { set_error("pipe mode: the pipe needs at least 5 cells along y"); return FS_INVALID_ARG; }
  PipeGeom& G = c->pipe;
  G.on = 1;
  G.a = p.pipe_radius;
  for (int g = 0; g < 4; ++g) {
    G.ox[g] = p.grid_min[0];
    G.hx[g] = d[0];
    G.oz[g] = p.grid_min[2];
    G.hz[g] = d[2];
  }
  G.ox[1] = p.grid_min[0] - 0.5 * d[0];
  G.hx[1] = ((p.grid_max[0] + 0.5 * d[0]) - (p.grid_min[0] - 0.5 * d[0])) / n[0];
  G.oz[3] = p.grid_min[2] - 0.5 * d[2];
  G.hz[3] = ((p.grid_max[2] + 0.5 * d[2]) - (p.grid_min[2] - 0.5 * d[2])) / n[2];
  // the WENO5 stencils of the cells inside the pipe must stay off the box's
  // ghost layers: three cells of the box around the pipe
  for (int k = 0; k < n[2]; ++k)
    for (int i = 0; i < n[0]; ++i) {
      const double X = G.ox[0] + i * G.hx[0], Z = G.oz[0] + k * G.hz[0];
      if (std::sqrt(X * X + Z * Z) - G.a <= 0.0 && (i < 3 || i > n[0] - 4 || k < 3 || k > n[2] - 4)) {
        set_error("pipe mode: the pipe must keep three cells of the box around it in x and z");
        c->pipe = PipeGeom{};
        return FS_INVALID_ARG;
      }
    }
  // the unknowns of the pressure system: every cell of a column inside the
  // pipe (wall distance <= 0, pipe_solid's test in the same rounding); the
  // first in the reference's row order (k, j, i) carries the deflation
  G.fi = G.fj = G.fk = -1;
  int64_t columns = 0;
  for (int k = 0; k < n[2]; ++k)
    for (int i = 0; i < n[0]; ++i) {
      const double X = G.ox[0] + i * G.hx[0], Z = G.oz[0] + k * G.hz[0];
      if (!(std::sqrt(X * X + Z * Z) - G.a > 0.0)) {
        if (G.fk < 0) { G.fi = i; G.fj = 0; G.fk = k; }
        ++columns;
      }
    }
  if (columns == 0) {
    set_error("pipe mode: no cell of the grid lies inside the pipe");
    c->pipe = PipeGeom{};
    return FS_INVALID_ARG;
  }
  G.cells = columns * n[1];
  return FS_OK;
}

// Operators of the box only: the pipe mode builds its level-set path, its
// ENO3 velocity advection, its body force and its projection, not yet its
// viscosity (and so neither its whole step).
fs_status box_only(const fs_ctx* c, const char* what) {
  if (!c->pipe.on) return FS_OK;
  set_error("%s is not built for the oil/water pipe mode (its viscosity is not built)", what);
  return FS_NOT_SUPPORTED;
}

// ---------------------------------------------------------------------------
// Krylov driver
// ---------------------------------------------------------------------------

// The loop control of a captured solve: before the loop it clears the batch
// counter and lets the loop start only if the solve is still running; after
// each batch of kGraphIters iterations it continues the loop while the solve
// runs and fewer than max_iter / kGraphIters + 2 batches have run (the
// bound that guarantees the loop ends whatever the state says).
__global__ void k_loop_start(cudaGraphConditionalHandle h, const PcgState* st, unsigned int* batches) {
  *batches = 0u;
  cudaGraphSetConditional(h, ((volatile const PcgState*)st)->done == 0 ? 1u : 0u);
}
__global__ void k_loop_next(cudaGraphConditionalHandle h, const PcgState* st, unsigned int* batches) {
  const volatile PcgState* vs = (volatile const PcgState*)st;
  const unsigned int n = *batches + 1u;
  *batches = n;
  const unsigned int cap = (unsigned int)(vs->max_iter / kGraphIters + 2);
  cudaGraphSetConditional(h, (vs->done == 0 && n < cap) ? 1u : 0u);
}

// Run the iterations of a solve until its state says stop (done != 0), as
// ONE graph launch: a captured CUDA graph whose conditional while node
// repeats a body of kGraphIters iterations plus the loop control above, so
// the host waits once per solve (or per reliable update of the mixed
// solve) instead of once per batch.  The graph is captured on first use per
// key (kernel arguments are baked into it).
template <class F>
fs_status drive_pcg(fs_ctx* c, std::pair<int, const void*> key, F&& enqueue_iteration, int max_iter, bool timed,
                    int kernels_per_iteration = 3) {
  if (c->prm.host_loop) {
    // the same batches launched from the host, the state polled after each;
    // bounded like the graph's loop
    const int cap = max_iter / kGraphIters + 2;
    int nb = 0;
    CK(cudaMemcpyAsync(c->st_host, c->st, sizeof(PcgState), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    while (!c->st_host->done && nb < cap) {
      for (int n = 0; n < kGraphIters; ++n) enqueue_iteration();
      CK(cudaGetLastError());
      ++nb;
      CK(cudaMemcpyAsync(c->st_host, c->st, sizeof(PcgState), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
    }
    c->launches += (int64_t)nb * kernels_per_iteration * kGraphIters;
    if (timed) c->pcg_launched_iterations += nb * kGraphIters;
    return FS_OK;
  }
  unsigned int* batches = c->tickets + 6;
  auto it = c->graphs.find(key);
  if (it == c->graphs.end()) {
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    // the loop start, then the while node
    CK(cudaStreamBeginCaptureToGraph(c->stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    k_loop_start<<<1, 1, 0, c->stream>>>(h, c->st, batches);
    CK(cudaStreamEndCapture(c->stream, &g));
    cudaGraphNode_t start = nullptr;
    size_t nroots = 1;
    CK(cudaGraphGetRootNodes(g, &start, &nroots));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t loop = nullptr;
    CK(cudaGraphAddNode(&loop, g, &start, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    for (int n = 0; n < kGraphIters; ++n) enqueue_iteration();
    k_loop_next<<<1, 1, 0, c->stream>>>(h, c->st, batches);
    CK(cudaStreamEndCapture(c->stream, &body));
    cudaGraphExec_t ge;
    CK(cudaGraphInstantiate(&ge, g, 0));
    cudaGraphDestroy(g);
    it = c->graphs.emplace(key, ge).first;
  }
  CK(cudaGraphLaunch(it->second, c->stream));
  CK(cudaMemcpyAsync(c->st_host, c->st, sizeof(PcgState), cudaMemcpyDeviceToHost, c->stream));
  unsigned int nb = 0;
  CK(cudaMemcpyAsync(c->sc_host + 15, batches, sizeof(unsigned int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::memcpy(&nb, c->sc_host + 15, sizeof nb);
  c->launches += 1 + (int64_t)nb * (kernels_per_iteration * kGraphIters + 1);
  if (timed) c->pcg_launched_iterations += (int)nb * kGraphIters;
  return FS_OK;
}

template <class V>
fs_status run_pcg(fs_ctx* c, int key, const Op7<V>& A, const V* b, V* x, V* r, V* p, V* q, double tol, int max_iter,
                  int criterion, int* iterations, double* rel, int* status) {
  PcgState init{};
  init.tol = tol;
  init.max_iter = max_iter;
  init.criterion = criterion;
  // FP32 viscosity solves can stall at their rounding floor before a tight tolerance
  init.stall_limit = (c->fp32 && key >= 100 && key < 110) ? 400 : 0;  // the FP32 forward viscosity solves
  *c->st_host = init;
  const bool timed = key < 100;  // pressure solves
  CK(cudaMemcpyAsync(c->st, c->st_host, sizeof(PcgState), cudaMemcpyHostToDevice, c->stream));
  if (timed) CK(cudaEventRecord(c->evp0, c->stream));
  pcg_init<V>(A, b, x, r, p, c->st, c->partials, c->stream);
  c->launches += 1;
  CK(cudaGetLastError());
  CKS(drive_pcg(c, std::make_pair(key, (const void*)nullptr),
                [&] { cg_iteration<V, V>(A, x, r, p, q, c->st, c->partials, c->stream); }, max_iter, timed));
  if (timed) {
    CK(cudaEventRecord(c->evp1, c->stream));
    CK(cudaEventSynchronize(c->evp1));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, c->evp0, c->evp1));
    c->pcg_ms += ms;
  }
  const PcgState& s = *c->st_host;
  if (iterations) *iterations = s.iter;
  if (rel) *rel = s.bb > 0 ? std::sqrt(s.rr / s.bb) : 0.0;
  if (status) *status = s.status;
  if (c->debug)
    std::fprintf(stderr, "[fs] pcg key %d: %d iterations, status %d, rel %.3e\n", key, s.iter, s.status,
                 s.bb > 0 ? std::sqrt(s.rr / s.bb) : 0.0);
  if (s.status == PCG_NONFINITE) {
    set_error("non-finite residual in a PCG solve (key %d, iteration %d)", key, s.iter);
    return FS_NONFINITE;
  }
  return FS_OK;
}

// ---------------------------------------------------------------------------
// operators, templated on the storage type S
// ---------------------------------------------------------------------------

template <class S>
S* F(void* p) { return static_cast<S*>(p); }

template <class S>
fs_status advect_levelset_t(fs_ctx* c, double dt, Tape* tp = nullptr) {
  const fs_params& P = c->prm;
  const double eps = P.weno_epsilon, dx = c->grid.dx;
  S *phi = F<S>(c->phi), *t1 = F<S>(c->s1), *t2 = F<S>(c->s2);
  S *u = F<S>(c->u), *v = F<S>(c->v), *w = F<S>(c->w);
  cudaStream_t s = c->stream;
  const PipeGeom* pg = c->pipe.on ? &c->pipe : nullptr;
  if (pg) {
    // the pipe's velocity set-up (ADVECTION_3D.h:380-490): u and w zeroed
    // outside the pipe, the ghost copies the update reads in the RK base
    // arrays, which the velocity stages fill only after the level set
    pipe_levelset_velocities<S>(u, v, w, F<S>(c->u0), F<S>(c->v0), F<S>(c->w0), c->Lu, c->Lv, c->Lw, *pg, s);
    u = F<S>(c->u0);
    v = F<S>(c->v0);
    w = F<S>(c->w0);
    c->launches += 3;
  }
  int stage = 0;
  auto fe = [&](S* src, const S* base, S* out, double c0, double c1) {
    if (tp && stage < 3)
      cudaMemcpyAsync(tp->ls[stage], src, c->Lc.total * c->S(), cudaMemcpyDeviceToDevice, s);
    ++stage;
    if (pg) fill_periodic_y<S>(src, c->Lc, s);
    else fill_extrap<S>(src, c->Lc, s);
    weno5_levelset<S>(src, base, out, u, v, w, c->Lc, c->Lu, c->Lv, c->Lw, dx, eps, dt, c0, c1, s, pg);
    c->launches += 2;
  };
  if (P.order == 3 && !(P.flags & FS_FLAG_LEVELSET_FORWARD_EULER)) {
    fe(phi, phi, t1, 0.0, 1.0);                        // phi1 = phi0 + dt L(phi0)
    fe(t1, phi, t2, 0.75, 0.25);                       // phi2 = 3/4 phi0 + 1/4 (phi1 + dt L(phi1))
    fe(t2, phi, t1, 1.0 / 3.0, 2.0 / 3.0);             // phi3 = 1/3 phi0 + 2/3 (phi2 + dt L(phi2))
  } else if (P.order == 3) {
    fe(phi, phi, t1, 0.0, 1.0);                        // the reference's order-3 level set: one Euler step
  } else {
    fe(phi, phi, t1, 0.0, 1.0);                        // Heun: phi1, then 1/2 phi0 + 1/2 (phi1 + dt L(phi1))
    fe(t1, phi, t2, 0.5, 0.5);
    std::swap(c->s1, c->s2);
  }
  std::swap(c->phi, c->s1);
  if (tp) CK(cudaMemcpyAsync(tp->ls[3], c->phi, c->Lc.total * c->S(), cudaMemcpyDeviceToDevice, s));
  CK(cudaGetLastError());
  return FS_OK;
}

// The WENO5 epsilon of the velocity advection (VELOCITY_ADVECTION.epsilon,
// ADVECTION_3D.h:112), which falls back to the level-set one when unset.
static double velocity_epsilon(const fs_ctx* c) {
  return c->prm.velocity_epsilon > 0.0 ? c->prm.velocity_epsilon : c->prm.weno_epsilon;
}

template <class S>
fs_status advect_velocity_t(fs_ctx* c, double dt) {
  const double eps = velocity_epsilon(c), dx = c->grid.dx;
  S *u = F<S>(c->u), *v = F<S>(c->v), *w = F<S>(c->w);
  if (c->pipe.on) {
    // the vertical pipe (ADVECTION_3D.h:244-358, the oil/water ENO3 path):
    // the ghost copies, then each component in place
    if (c->prm.velocity_scheme != FS_VELOCITY_ENO3) {
      set_error("the pipe mode advects the velocity with ENO3 (use_3rd_eno_v) only");
      return FS_NOT_SUPPORTED;
    }
    S* comps[3] = {u, v, w};
    const Lay* lays[3] = {&c->Lu, &c->Lv, &c->Lw};
    S* gen[3] = {F<S>(c->pgen[0]), F<S>(c->pgen[1]), F<S>(c->pgen[2])};
    S* gx[3] = {F<S>(c->pgx[0]), F<S>(c->pgx[1]), F<S>(c->pgx[2])};
    S* gz[3] = {F<S>(c->pgz[0]), F<S>(c->pgz[1]), F<S>(c->pgz[2])};
    c->launches += pipe_velocity_copies<S>(comps, gen, gx, gz, lays, c->pipe, c->stream);
    for (int a = 0; a < 3; ++a)
      eno3_pipe<S>(comps[a], gen[a], gx[a], gz[a], gen[0], gen[1], gen[2], c->Lc, c->Lu, c->Lv, c->Lw, a, c->pipe,
                   dx, dt, c->stream);
    c->launches += 3;
    CK(cudaGetLastError());
    return FS_OK;
  }
  if (c->prm.velocity_scheme == FS_VELOCITY_ENO3) {
    eno3_mac<S>(u, F<S>(c->ua), u, v, w, c->Lu, c->Lu, c->Lv, c->Lw, 0, dx, dt, c->stream);
    eno3_mac<S>(v, F<S>(c->va), u, v, w, c->Lv, c->Lu, c->Lv, c->Lw, 1, dx, dt, c->stream);
    eno3_mac<S>(w, F<S>(c->wa), u, v, w, c->Lw, c->Lu, c->Lv, c->Lw, 2, dx, dt, c->stream);
  } else {
    weno5_mac<S>(u, F<S>(c->ua), u, v, w, c->Lu, c->Lu, c->Lv, c->Lw, 0, dx, eps, dt, c->stream);
    weno5_mac<S>(v, F<S>(c->va), u, v, w, c->Lv, c->Lu, c->Lv, c->Lw, 1, dx, eps, dt, c->stream);
    weno5_mac<S>(w, F<S>(c->wa), u, v, w, c->Lw, c->Lu, c->Lv, c->Lw, 2, dx, eps, dt, c->stream);
  }
  c->launches += 3;
  std::swap(c->u, c->ua);
  std::swap(c->v, c->va);
  std::swap(c->w, c->wa);
  CK(cudaGetLastError());
  return FS_OK;
}

// One reinitialisation block from `in` into `out` (out may be `base`):
// S from `in`, reinit_iterations pseudo-steps, the last one combined as
// c0*base + c1*result.
// Fast sweeping of `in` into `out` (EULERIAN_FLUID_SOLVER_3D.h:2202-2205:
// LEVELSET_3D::ReinitializeByFastSweeping); direction < 0 takes the
// context's counter and advances it.
template <class S>
fs_status fast_sweeping_t(fs_ctx* c, const void* in, void* out, int direction, int pairs) {
  const bool typo = (c->prm.flags & FS_FLAG_SORT_TYPO) != 0;
  if (direction < 0) direction = c->sweep_direction++;
  if (typo) CK(cudaMemsetAsync(c->fsflag, 0, sizeof(int), c->stream));
  c->launches += fast_sweeping<S>(F<S>(const_cast<void*>(in)), F<S>(out), c->fsfixed, c->Lc, c->grid.dx, direction,
                                  pairs, typo ? 1 : 0, c->fsflag, c->stream);
  CK(cudaGetLastError());
  if (typo) {
    int flag = 0;
    CK(cudaMemcpyAsync(&flag, c->fsflag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (flag) {
      set_error("the reference's sort reads its uninitialised a2 on this input (FS_FLAG_SORT_TYPO)");
      return FS_NONFINITE;
    }
  }
  return FS_OK;
}

template <class S>
fs_status reinit_block_t(fs_ctx* c, void* in, void* out, void* base, double c0, double c1, void* scrA, void* scrB,
                         std::vector<void*>* tape = nullptr) {
  const fs_params& P = c->prm;
  const double dx = c->grid.dx, dtau = dx / P.reinit_scaling;
  const int n = P.reinit_iterations;
  cudaStream_t s = c->stream;
  if (P.fast_sweeping) {
    // the sweeps first, into scratch (in may be the RK base)
    CKS(fast_sweeping_t<S>(c, in, scrA, -1, 1));
    in = scrA;
  }
  if (n == 0) {
    if (c0 != 0.0) { axpby<S>(F<S>(out), F<S>(base), F<S>(in), c0, c1, c->Lc, s); c->launches += 1; }
    else if (out != in) CK(cudaMemcpyAsync(out, in, c->Lc.total * c->S(), cudaMemcpyDeviceToDevice, s));
    return FS_OK;
  }
  sign_function<S>(F<S>(in), F<S>(c->sgn), c->Lc, dx, s);
  c->launches += 1 + 2 * n;
  void* cur = in;
  for (int it = 0; it < n; ++it) {
    const bool last = it == n - 1;
    void* dst = last ? out : (cur == scrA ? scrB : scrA);
    if (tape) CK(cudaMemcpyAsync((*tape)[it], cur, c->Lc.total * c->S(), cudaMemcpyDeviceToDevice, s));
    if (c->pipe.on) fill_periodic_y<S>(F<S>(cur), c->Lc, s);  // ADVECTION_3D.h:360-378
    else fill_extrap<S>(F<S>(cur), c->Lc, s);
    sussman_step<S>(F<S>(cur), F<S>(c->sgn), F<S>(base), F<S>(dst), c->Lc, dx, P.weno_epsilon, dtau,
                    last ? c0 : 0.0, last ? c1 : 1.0, (P.flags & FS_FLAG_REINIT_TYPO) ? 1 : 0, s);
    cur = dst;
  }
  CK(cudaGetLastError());
  return FS_OK;
}

template <class S>
fs_status reinitialize_t(fs_ctx* c, Tape* tp = nullptr) {
  // RK combination of reinitialisation blocks (EULERIAN_FLUID_SOLVER_3D.h:959-979, 1081-1109)
  if (c->prm.order == 3) {
    CKS(reinit_block_t<S>(c, c->phi, c->s1, c->phi, 0.0, 1.0, c->s2, c->s3, tp ? &tp->re[0] : nullptr));
    CKS(reinit_block_t<S>(c, c->s1, c->s4, c->phi, 0.75, 0.25, c->s2, c->s3, tp ? &tp->re[1] : nullptr));
    CKS(reinit_block_t<S>(c, c->s4, c->phi, c->phi, 1.0 / 3.0, 2.0 / 3.0, c->s2, c->s3, tp ? &tp->re[2] : nullptr));
  } else {
    CKS(reinit_block_t<S>(c, c->phi, c->s1, c->phi, 0.0, 1.0, c->s2, c->s3, tp ? &tp->re[0] : nullptr));
    CKS(reinit_block_t<S>(c, c->s1, c->phi, c->phi, 0.5, 0.5, c->s2, c->s3, tp ? &tp->re[1] : nullptr));
  }
  return FS_OK;
}

template <class S>
fs_status viscosity_t(fs_ctx* c, double dt, int* iters_out) {
  const fs_params& P = c->prm;
  if (!P.viscosity) {
    if (iters_out) *iters_out = 0;
    return FS_OK;
  }
  if (P.viscosity == 2) {
    // the reference's air/water explicit update (VISCOSITY_3D.h:452-563)
    const int in_place = (P.flags & FS_FLAG_VISCOSITY_IN_PLACE) ? 1 : 0;
    c->launches += viscosity_explicit<S>(F<S>(c->phi), F<S>(c->u), F<S>(c->v), F<S>(c->w), F<S>(c->ua), F<S>(c->va),
                                         F<S>(c->wa), c->Lc, c->Lu, c->Lv, c->Lw, c->grid.dx, dt, P.rho_neg,
                                         P.rho_pos, P.mu_neg, P.mu_pos, in_place, c->stream);
    if (!in_place) {
      std::swap(c->u, c->ua);
      std::swap(c->v, c->va);
      std::swap(c->w, c->wa);
    }
    CK(cudaGetLastError());
    if (iters_out) *iters_out = 0;
    return FS_OK;
  }
  const Lay* lays[3] = {&c->Lu, &c->Lv, &c->Lw};
  void* comps[3] = {c->u, c->v, c->w};
  // all three systems from the pre-viscosity velocities
  for (int a = 0; a < 3; ++a) {
    viscosity_system<S>(F<S>(c->phi), F<S>(c->u), F<S>(c->v), F<S>(c->w), c->Lc, c->Lu, c->Lv, c->Lw, a,
                        c->grid.dx, dt, P.rho_neg, P.rho_pos, P.mu_neg, P.mu_pos, F<S>(c->vs[a][0]),
                        F<S>(c->vs[a][1]), F<S>(c->vs[a][2]), F<S>(c->vs[a][3]), F<S>(c->vs[a][4]), c->stream);
    c->launches += 1;
    CK(cudaMemcpyAsync(c->vs[a][5], comps[a], lays[a]->total * c->S(), cudaMemcpyDeviceToDevice, c->stream));
  }
  CK(cudaGetLastError());
  int total = 0;
  for (int a = 0; a < 3; ++a) {
    Op7<S> A{F<S>(c->vs[a][0]), F<S>(c->vs[a][1]), F<S>(c->vs[a][2]), F<S>(c->vs[a][3]), *lays[a]};
    int it = 0, st = 0;
    CKS(run_pcg<S>(c, 100 + a, A, F<S>(c->vs[a][4]), F<S>(c->vs[a][5]), F<S>(c->vs[a][6]), F<S>(c->vs[a][7]),
                   F<S>(c->vs[a][8]), P.viscosity_tolerance, P.viscosity_max_iteration, FS_STOP_RELATIVE, &it,
                   nullptr, &st));
    total += it;
  }
  // the solution buffers stay where the captured solver graphs expect them;
  // copy the result back into the velocity fields
  for (int a = 0; a < 3; ++a)
    CK(cudaMemcpyAsync(comps[a], c->vs[a][5], lays[a]->total * c->S(), cudaMemcpyDeviceToDevice, c->stream));
  if (iters_out) *iters_out = total;
  return FS_OK;
}

// The FP32 + FP64 defect-correction solve of A(phi) x = b (A the pressure
// operator evaluated from phi, b and x FP64 cell fields): the projection's
// solve and, in FP32 contexts, the adjoint's transposed solve with the same
// symmetric operator.  *iters, *outer, *rel and *st report the Krylov
// iterations, the defect corrections, the final relative FP64 residual and
// the PCG status.
template <class S>
fs_status mixed_solve(fs_ctx* c, S* phi, double* b, double* x, int* iters_out, int* outer_out, double* rel_out,
                      int* st_out) {
  const fs_params& P = c->prm;
  const double dx = c->grid.dx;
  cudaStream_t s = c->stream;
  int iters = 0, outer = 0, st = 0;
  double rel = 0.0;
  const bool rb = c->red_black;
  build_pressure_operator<S, float>(phi, c->Lc, dx, P.rho_neg, P.rho_pos, (float*)c->pax, (float*)c->pay,
                                    (float*)c->paz, (float*)c->pdiag, c->scalars + 12, deflate(c), s,
                                    (c->lean || rb) ? c->pdinv : nullptr, pipe_of(c));
  Op7<float> A{(float*)c->pax, (float*)c->pay, (float*)c->paz, (float*)c->pdiag, c->Lc, 1, c->scalars + 12};
  A.c_extra = deflated_cell(c);
  A.flux32 = c->flux32;
  if (c->lean) A.dinv16 = c->pdinv;
  // red-black: the black Schur complement on the packed half layout, its
  // Jacobi preconditioner bf16 1/diag(S) (IC(0) in red-black order) or the
  // black cells' own bf16 1/diag
  RbOp R{(float*)c->pax, (float*)c->pay, (float*)c->paz, c->Lc, c->Lh, c->scalars + 12};
  Op7<float> Ah{nullptr, nullptr, nullptr, nullptr, c->Lh};
  Ah.dinv16 = c->rb_dinv;
  if (rb) {
    if (c->rb_ic0)
      rb_schur_dinv(R, c->rb_dinv, s);
    else
      rb_gather<unsigned short, unsigned short>(c->pdinv, c->rb_dinv, c->Lc, c->Lh, s);
    rb_gather<double, double>(x, c->rb_x, c->Lc, c->Lh, s);  // the initial guess's black cells
    c->launches += 2;
  }
  double bb = 0.0;
  float *r32 = (float*)c->pr, *p32 = (float*)c->pp, *q32 = (float*)c->pq;
  // the Krylov vectors of the chosen form
  float* kr = rb ? c->rb_r : r32;
  float* kp = rb ? c->rb_p : p32;
  const Op7<float>& KA = rb ? Ah : A;
  // red-black: p64 <- the black iterate, red cells eliminated in FP64
  auto commit = [&]() {
    if (!rb) return;
    rb_commit<S>(phi, c->rb_x, b, x, c->Lc, c->Lh, dx, P.rho_neg, P.rho_pos, deflate(c), s);
    c->launches += 1;
  };
  // true FP64 residual b - A64 p64 with A64 evaluated from phi in FP64; its
  // FP32 image lands in r32 (red-black: its black cells in the packed
  // residual), the Krylov residual of the mixed solve
  auto defect = [&](const float* x32, double* rel_out) -> fs_status {
    defect_residual<S>(phi, x, x32, b, nullptr, r32, c->Lc, dx, P.rho_neg, P.rho_pos, c->partials,
                       c->tickets + 2, c->scalars + 2, deflate(c), s, pipe_of(c));
    c->launches += 1;
    if (rb) {
      rb_gather<float, float>(r32, c->rb_r, c->Lc, c->Lh, s);
      c->launches += 1;
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->sc_host, c->scalars, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    bb = c->sc_host[1];
    const double rr = c->sc_host[2];
    *rel_out = bb > 0 ? std::sqrt(rr / bb) : 0.0;
    outer += 1;
    if (!std::isfinite(*rel_out) && !x32) {
      set_error("non-finite defect residual");
      return FS_NONFINITE;
    }
    return FS_OK;
  };
  commit();
  CKS(defect(nullptr, &rel));
  st = PCG_CONVERGED;
  if (rel > P.tolerance) {
    // Mixed-precision CG: the FP64 pressure p64 (red-black: its black cells,
    // packed) is the iterate; the face couplings, the residual r, the
    // search direction p and q = A p are FP32 (the flux-form operator in
    // FP32 arithmetic, Op7::flux32, or the red-black Schur complement in
    // its offset form) and the Jacobi preconditioner is 1/diag in bf16: 64
    // bytes per unknown and iteration (red-black: 56 per cell at half the
    // iterations) against 120 for the FP64 solve.  Every time the recursive
    // residual drops by reliable_delta the true FP64 residual of p64
    // replaces it (reliable update), keeping the search direction; the
    // recursion stops at the tolerance itself and the true residual
    // decides.  A sequence whose true residual got worse is rolled back to
    // the last accepted pressure and restarted.
    const size_t pbytes = c->Lc.total * sizeof(double);
    CK(cudaMemcpyAsync(c->p64bak, x, pbytes, cudaMemcpyDeviceToDevice, s));
    PcgState init{};
    init.criterion = 2;  // absolute 2-norm of the recursive residual, in b's units
    init.tol = P.tolerance * std::sqrt(bb);
    init.max_iter = P.max_iteration;
    init.reliable_delta = c->reliable_delta;
    init.bb = bb;  // ||b||^2 of the pressure system, for the recursive relative residual
    *c->st_host = init;
    CK(cudaMemcpyAsync(c->st, c->st_host, sizeof(PcgState), cudaMemcpyHostToDevice, s));
    CK(cudaEventRecord(c->evp0, s));
    // the residual already holds the image of b - A p64: start the recursion from it
    pcg_resume<float, float>(KA, kr, kp, c->st, c->partials, 1, s);
    c->launches += 2;
    int failures = 0, passes = 0;
    double best = rel;
    for (;;) {
      ++passes;  // each pass runs at least one iteration or ends the solve; this bounds the host loop too
      if (rb) {
        CKS(drive_pcg(c, std::make_pair(4, (const void*)nullptr),
                      [&] {
                        rb_iteration(R, Ah, c->rb_x, c->rb_r, c->rb_p, c->rb_q, c->rb_tau, c->st, c->partials, s);
                      },
                      P.max_iteration, true, 4));
      } else {
        CKS(drive_pcg(c, std::make_pair(2, (const void*)x),
                      [&] { cg_iteration<float, double>(A, x, r32, p32, q32, c->st, c->partials, s); },
                      P.max_iteration, true));
      }
      const int status = c->st_host->status;
      iters = c->st_host->iter;
      const double recursive = c->st_host->bb > 0 ? std::sqrt(c->st_host->rr / c->st_host->bb) : 0.0;
      double now = 0.0;
      commit();
      CKS(defect(nullptr, &now));  // residual <- true residual of the current pressure
      bool restart = false;
      if (!std::isfinite(now) || now > 100.0 * best) {
        // diverged (not a CG residual oscillation): back to the best pressure
        CK(cudaMemcpyAsync(x, c->p64bak, pbytes, cudaMemcpyDeviceToDevice, s));
        if (rb) {
          rb_gather<double, double>(x, c->rb_x, c->Lc, c->Lh, s);
          c->launches += 1;
        }
        CKS(defect(nullptr, &now));
        restart = true;
        ++failures;
      } else {
        if (now < best) {
          best = now;
          CK(cudaMemcpyAsync(c->p64bak, x, pbytes, cudaMemcpyDeviceToDevice, s));
        }
        // restart the direction after a breakdown or when the recursion
        // has drifted far from the true residual
        restart = status == PCG_STAGNATED || now > 10.0 * recursive;
      }
      rel = now;
      if (c->debug)
        std::fprintf(stderr, "[fs] mixed solve%s: iteration %d, status %d, recursive %.3e, true %.3e, best %.3e%s\n",
                     rb ? " (red-black)" : "", iters, status, recursive, now, best, restart ? ", restart" : "");
      if (now <= P.tolerance) { st = PCG_CONVERGED; break; }
      if (iters >= P.max_iteration || failures > 8 || passes > P.max_iteration + 8) {
        // leave the best pressure found
        CK(cudaMemcpyAsync(x, c->p64bak, pbytes, cudaMemcpyDeviceToDevice, s));
        rel = best;
        st = PCG_MAXITER;
        break;
      }
      pcg_resume<float, float>(KA, kr, kp, c->st, c->partials, restart ? 1 : 0, s);
      c->launches += 2;
      CK(cudaGetLastError());
    }
    CK(cudaEventRecord(c->evp1, s));
    CK(cudaEventSynchronize(c->evp1));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, c->evp0, c->evp1));
    c->pcg_ms += ms;
  }
  *iters_out = iters;
  *outer_out = outer;
  *rel_out = rel;
  *st_out = st;
  return FS_OK;
}

// PROJECTION_3D::Solve; c0/c1 fuse the RK combination with base (u0, v0, w0)
template <class S>
fs_status project_t(fs_ctx* c, double dt, double c0, double c1, fs_solve_report* rep) {
  const fs_params& P = c->prm;
  const double dx = c->grid.dx;
  cudaStream_t s = c->stream;
  const bool faithful = (P.flags & FS_FLAG_FAITHFUL_PROJECTION) != 0;
  const bool pipe = c->pipe.on != 0;
  S *u = F<S>(c->u), *v = F<S>(c->v), *w = F<S>(c->w), *phi = F<S>(c->phi);
  if (pipe) {
    // the vertical pipe (PROJECTION_3D.h:416-441 with oil_water_simulation):
    // the divergence of the pipe's velocity copies on the cells inside it
    pipe_divergence_rhs<S>(u, v, w, c->Lc, c->Lu, c->Lv, c->Lw, c->pipe, dx, dt, c->b64, c->div64, c->partials,
                           c->tickets + 0, c->scalars + 0, s);
  } else {
    divergence_rhs<S>(u, v, w, c->Lc, c->Lu, c->Lv, c->Lw, dx, dt, c->b64, c->div64, c->partials, c->tickets + 0,
                      c->scalars + 0, s);
  }
  // surface tension: curvature, jc = sigma kappa, and the jump terms of the
  // right-hand side (DetermineJumpConditionField, PROJECTION_3D.h:746-792);
  // the pipe's dimensionless form always carries jc = kappa/We (:758-762)
  const double sigma = pipe ? 1.0 / P.pipe_We : P.surface_tension;
  const double* kap = nullptr;
  if (sigma != 0.0) {
    fill_extrap<S>(phi, c->Lc, s);  // the curvature's ghost fill (LEVELSET_3D.h:999), the pipe's too
    curvature<S>(phi, c->kappa, c->Lc, dx, (P.flags & FS_FLAG_CURVATURE_TYPO) ? 1 : 0, c->scalars + 13, s);
    jump_rhs<S>(phi, c->kappa, sigma, c->b64, c->Lc, dx, P.rho_neg, P.rho_pos, faithful ? 1 : 0, c->partials,
                c->tickets + 5, c->scalars + 0, s, pipe_of(c));
    kap = c->kappa;
    c->launches += 3;
  }
  subtract_mean(c->b64, c->Lc, c->scalars + 0, c->partials, c->tickets + 1, c->scalars + 1, s, pipe_of(c));
  c->launches += 4;  // divergence, mean, pressure faces, pressure diagonal
  CK(cudaGetLastError());
  int iters = 0, outer = 0, st = 0;
  double rel = 0.0;
  if (!c->fp32) {
    build_pressure_operator<S, double>(phi, c->Lc, dx, P.rho_neg, P.rho_pos, (double*)c->pax, (double*)c->pay,
                                       (double*)c->paz, (double*)c->pdiag, c->scalars + 12, deflate(c), s, nullptr,
                                       pipe_of(c));
    Op7<double> A{(double*)c->pax, (double*)c->pay, (double*)c->paz, (double*)c->pdiag, c->Lc, 1, c->scalars + 12};
    A.c_extra = deflated_cell(c);
    CKS(run_pcg<double>(c, 1, A, c->b64, c->p64, (double*)c->pr, (double*)c->pp, (double*)c->pq, P.tolerance,
                        P.max_iteration, P.stop, &iters, &rel, &st));
    outer = 1;
  } else {
    CKS(mixed_solve<S>(c, phi, c->b64, c->p64, &iters, &outer, &rel, &st));
  }
  if (pipe) {
    // the pipe's velocity update and periodic rows (PROJECTION_3D.h:1099-1449);
    // the RK combination, if any, is the caller's
    pipe_velocity_correct<S>(u, v, w, c->p64, phi, c->kappa, c->Lc, c->Lu, c->Lv, c->Lw, c->pipe, dx, dt, P.rho_neg,
                             P.rho_pos, sigma, s);
    c->launches += 4;
  } else {
    velocity_correct<S>(u, F<S>(c->u0), c->p64, phi, c->Lu, c->Lc, 0, dx, dt, P.rho_neg, P.rho_pos, faithful, c0, c1,
                        kap, sigma, s);
    velocity_correct<S>(v, F<S>(c->v0), c->p64, phi, c->Lv, c->Lc, 1, dx, dt, P.rho_neg, P.rho_pos, faithful, c0, c1,
                        kap, sigma, s);
    velocity_correct<S>(w, F<S>(c->w0), c->p64, phi, c->Lw, c->Lc, 2, dx, dt, P.rho_neg, P.rho_pos, faithful, c0, c1,
                        kap, sigma, s);
    c->launches += 3;
  }
  CK(cudaGetLastError());
  if (rep) {
    divergence_norms<S>(u, v, w, c->Lc, c->Lu, c->Lv, c->Lw, dx, c->partials, c->tickets + 3, c->scalars + 4, s);
    c->launches += 1;
    CK(cudaMemcpyAsync(c->sc_host, c->scalars, 8 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    rep->iterations = iters;
    rep->outer_iterations = outer;
    rep->rel_residual = rel;
    rep->rz = c->st_host->rz;
    rep->div_l2 = std::sqrt(c->sc_host[4]);
    rep->div_linf = c->sc_host[5];
  }
  if (st == PCG_MAXITER) {
    set_error("pressure solve stopped at its iteration cap (relative residual %.3e)", rel);
    return FS_NOT_CONVERGED;
  }
  return FS_OK;
}

template <class S>
fs_status gravity_t(fs_ctx* c, double dt) {
  const double* g = c->prm.gravity;
  if (c->pipe.on) {
    // the vertical pipe's dimensionless body force (EULERIAN_FLUID_SOLVER_3D.h:2304-2326)
    const fs_params& P = c->prm;
    const double dy = (P.grid_max[1] - P.grid_min[1]) / (c->grid.ny - 1);
    fill_periodic_y<S>(F<S>(c->phi), c->Lc, c->stream);
    pipe_forcing<S>(F<S>(c->v), F<S>(c->phi), c->Lv, c->Lc, c->pipe, P.pipe_R1 / (P.pipe_V0 * P.pipe_V0),
                    dt * g[1], dt * P.pipe_f, P.pipe_oil_density, P.pipe_eta, 1.5 * dy, c->stream);
    c->launches += 2;
    CK(cudaGetLastError());
    return FS_OK;
  }
  const Lay* lays[3] = {&c->Lu, &c->Lv, &c->Lw};
  void* comps[3] = {c->u, c->v, c->w};
  for (int a = 0; a < 3; ++a)
    if (g[a] != 0.0) { add_const_faces<S>(F<S>(comps[a]), *lays[a], a, dt * g[a], 1, c->stream); c->launches += 1; }
  CK(cudaGetLastError());
  return FS_OK;
}

// One SolveForRK stage (EULERIAN_FLUID_SOLVER_3D.h:1453-1476): advection,
// gravity, viscosity, projection; the projection's velocity update also
// applies the stage's RK combination with the step's initial velocity.
// copy the three velocity components into a tape slot
fs_status tape_velocity(fs_ctx* c, void* const dst[3]) {
  const Lay* lays[3] = {&c->Lu, &c->Lv, &c->Lw};
  void* comps[3] = {c->u, c->v, c->w};
  for (int a = 0; a < 3; ++a)
    CK(cudaMemcpyAsync(dst[a], comps[a], lays[a]->total * c->S(), cudaMemcpyDeviceToDevice, c->stream));
  return FS_OK;
}

template <class S>
fs_status stage_t(fs_ctx* c, double dt, double c0, double c1, fs_step_report* rep, Tape* tp = nullptr,
                  int stage = 0) {
  if (tp) CKS(tape_velocity(c, tp->vel[stage][0]));
  CKS(advect_velocity_t<S>(c, dt));
  const Lay* lays[3] = {&c->Lu, &c->Lv, &c->Lw};
  if (!(c->prm.flags & FS_FLAG_FAITHFUL_PROJECTION) && !c->pipe.on) {
    // no penetration: advection also updates the wall faces, which hold zero
    zero_walls<S>(F<S>(c->u), *lays[0], 0, c->stream);
    zero_walls<S>(F<S>(c->v), *lays[1], 1, c->stream);
    zero_walls<S>(F<S>(c->w), *lays[2], 2, c->stream);
    c->launches += 3;
  }
  CKS(gravity_t<S>(c, dt));
  if (tp) CKS(tape_velocity(c, tp->vel[stage][1]));
  int vit = 0;
  CKS(viscosity_t<S>(c, dt, &vit));
  if (tp) CKS(tape_velocity(c, tp->vel[stage][2]));
  fs_solve_report pr{};
  fs_status st = project_t<S>(c, dt, c0, c1, &pr);
  if (st != FS_OK && st != FS_NOT_CONVERGED) return st;
  if (c->pipe.on && c0 != 0.0) {
    // the pipe's projection leaves the RK combination to its caller
    // (EULERIAN_FLUID_SOLVER_3D.h:938-955: c0 u_rk + c1 u on every face)
    void* comps[3] = {c->u, c->v, c->w};
    void* base[3] = {c->u0, c->v0, c->w0};
    for (int a = 0; a < 3; ++a) axpby<S>(F<S>(comps[a]), F<S>(base[a]), F<S>(comps[a]), c0, c1, *lays[a], c->stream);
    c->launches += 3;
    CK(cudaGetLastError());
  }
  if (tp) CK(cudaMemcpyAsync(tp->p[stage], c->p64, c->Lc.total * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  if (rep) {
    rep->pcg_iterations += pr.iterations;
    rep->outer_iterations += pr.outer_iterations;
    rep->viscosity_iterations += vit;
    rep->projections += 1;
    rep->max_rel_residual = std::max(rep->max_rel_residual, pr.rel_residual);
    rep->div_l2 = pr.div_l2;
    rep->div_linf = pr.div_linf;
  }
  return st;
}

template <class S>
fs_status step_t(fs_ctx* c, double dt, fs_step_report* rep, Tape* tp = nullptr) {
  const int order = c->prm.order;
  fs_status worst = FS_OK;
  CKS(advect_levelset_t<S>(c, dt, tp));
  const size_t bu = c->Lu.total * c->S(), bv = c->Lv.total * c->S(), bw = c->Lw.total * c->S();
  if (order > 1) {
    CK(cudaMemcpyAsync(c->u0, c->u, bu, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->v0, c->v, bv, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->w0, c->w, bw, cudaMemcpyDeviceToDevice, c->stream));
  }
  int stage_index = 0;
  auto stage = [&](double c0, double c1) -> fs_status {
    fs_status s = stage_t<S>(c, dt, c0, c1, rep, tp, stage_index++);
    if (s == FS_NOT_CONVERGED) { worst = s; return FS_OK; }
    return s;
  };
  if (order == 1) {
    CKS(stage(0.0, 1.0));
  } else if (order == 2) {
    CKS(stage(0.0, 1.0));
    CKS(stage(0.5, 0.5));
  } else {
    CKS(stage(0.0, 1.0));
    CKS(stage(0.75, 0.25));
    CKS(stage(1.0 / 3.0, 2.0 / 3.0));
  }
  CKS(reinitialize_t<S>(c, tp));
  return worst;
}

template <class S>
fs_status curvature_t(fs_ctx* c) {
  const fs_params& P = c->prm;
  fill_extrap<S>(F<S>(c->phi), c->Lc, c->stream);
  curvature<S>(F<S>(c->phi), c->kappa, c->Lc, c->grid.dx, (P.flags & FS_FLAG_CURVATURE_TYPO) ? 1 : 0,
               c->scalars + 13, c->stream);
  c->launches += 2;
  CK(cudaGetLastError());
  return FS_OK;
}

template <class S>
fs_status cfl_t(fs_ctx* c, double* dt) {
  absmax3<S>(F<S>(c->u), F<S>(c->v), F<S>(c->w), c->Lu, c->Lv, c->Lw, c->scalars + 8, c->stream);
  c->launches += 3;
  if (c->prm.surface_tension != 0.0 || c->pipe.on) CKS(curvature_t<S>(c));
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c->sc_host + 8, c->scalars + 8, 6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const fs_params& P = c->prm;
  if (c->pipe.on) {
    // the pipe's dimensionless form with the semi-implicit viscosity
    // (EULERIAN_FLUID_SOLVER_3D.h:2673-2785): each velocity's maximum over
    // the spacing of its own face grid, the body force's term with R1/V0^2
    // and f, the surface term with 1/We and min(water/oil, 1), no viscous
    // term.  The curvature maximum is that of the current level set (the
    // reference reads the one its last projection computed).
    const PipeGeom& G = c->pipe;
    const int ny = c->grid.ny;
    const double d1 = (P.grid_max[1] - P.grid_min[1]) / (ny - 1);
    const double hv = ((P.grid_max[1] + 0.5 * d1) - (P.grid_min[1] - 0.5 * d1)) / ny;  // dy of the v faces
    const double hu = G.hx[1], hw = G.hz[3];
    const double c_f = (c->sc_host[8] * (1.0 / hu) + c->sc_host[9] * (1.0 / hv)) + c->sc_host[10] * (1.0 / hw);
    const double rho_min = std::min(P.pipe_oil_density, P.pipe_oil_density * P.rho_pos);  // min(oil, water)
    const double g_f = std::sqrt(P.pipe_R1 / (P.pipe_V0 * P.pipe_V0) *
                                 (std::fabs(P.gravity[1]) + std::fabs(1.0 / rho_min * P.pipe_f)) * (1.0 / hv));
    const double h = std::min(std::min(hu, hv), hw);
    const double s_f = std::sqrt(((1.0 / P.pipe_We) * c->sc_host[13]) / (std::min(P.rho_pos, 1.0) * (h * h)));
    const double cv = c_f + 0.0;
    const double cfl = 0.5 * (cv + std::sqrt((cv * cv + 4.0 * (g_f * g_f)) + 4.0 * (s_f * s_f)));
    *dt = P.cfl / cfl;
    return FS_OK;
  }
  const double inv = 1.0 / c->grid.dx, inv2 = 1.0 / (c->grid.dx * c->grid.dx);
  const double c_f = (c->sc_host[8] * inv + c->sc_host[9] * inv) + c->sc_host[10] * inv;
  const double g_f = std::sqrt(std::fabs(P.gravity[1]) * inv);
  // semi-implicit viscosity imposes no limit; explicit (off) uses the reference's term
  // semi-implicit viscosity imposes no limit; otherwise the reference's
  // air/water term (EULERIAN_FLUID_SOLVER_3D.h:2765-2768)
  const double nu = P.viscosity == 1 ? 0.0 : std::max(P.mu_neg / P.rho_neg, P.mu_pos / P.rho_pos);
  const double v_f = nu * ((2.0 * inv2 + 2.0 * inv2) + 2.0 * inv2);
  // surface tension (EULERIAN_FLUID_SOLVER_3D.h:2741-2745): sqrt(sigma kappa_max / (min rho dx^2))
  const double s_f = P.surface_tension != 0.0
                         ? std::sqrt((P.surface_tension * c->sc_host[13]) /
                                     (std::min(P.rho_neg, P.rho_pos) * (c->grid.dx * c->grid.dx)))
                         : 0.0;
  const double cv = c_f + v_f;
  const double cfl = 0.5 * (cv + std::sqrt((cv * cv + 4.0 * (g_f * g_f)) + 4.0 * (s_f * s_f)));
  *dt = P.cfl / cfl;
  return FS_OK;
}

// ---------------------------------------------------------------------------
// Adjoint of the timestep (FP64 contexts)
// ---------------------------------------------------------------------------

// Buffers of the adjoint, allocated on first use.
fs_status adj_alloc(fs_ctx* c) {
  if (c->abar[0]) return FS_OK;
  const size_t cb = c->Lc.total * sizeof(double);
  const size_t fb[3] = {c->Lu.total * sizeof(double), c->Lv.total * sizeof(double), c->Lw.total * sizeof(double)};
  CKS(dalloc(c, (void**)&c->abar[0], cb));
  for (int a = 0; a < 3; ++a) CKS(dalloc(c, (void**)&c->abar[1 + a], fb[a]));
  for (double*& p : c->awork_c) CKS(dalloc(c, (void**)&p, cb));
  for (auto& t : c->awork_f)
    for (int a = 0; a < 3; ++a) CKS(dalloc(c, (void**)&t[a], fb[a]));
  for (int a = 0; a < 3; ++a) {
    CKS(dalloc(c, (void**)&c->a_vlam[a], fb[a]));
    CKS(dalloc(c, (void**)&c->a_vxb[a], fb[a]));
  }
  CKS(dalloc(c, (void**)&c->a_rho, 4 * sizeof(double)));
  if (!c->fp32) {
    c->a_ax = (double*)c->pax; c->a_ay = (double*)c->pay; c->a_az = (double*)c->paz; c->a_diag = (double*)c->pdiag;
    c->a_r = (double*)c->pr; c->a_p = (double*)c->pp; c->a_q = (double*)c->pq;
    for (int a = 0; a < 3; ++a)
      for (int m = 0; m < 9; ++m) c->a_vs[a][m] = (double*)c->vs[a][m];
  } else {
    // FP32 contexts: the transposed pressure solve reuses the forward's
    // FP32 + FP64 refinement machinery; only the viscosity systems need FP64
    // buffers of their own
    if (c->prm.viscosity == 1) {
      const size_t fmax = std::max(fb[0], std::max(fb[1], fb[2]));
      for (int m = 0; m < 9; ++m) {
        CKS(dalloc(c, (void**)&c->a_vs[0][m], fmax));
        c->a_vs[1][m] = c->a_vs[2][m] = c->a_vs[0][m];
      }
    }
  }
  return FS_OK;
}

// Tape buffers for one step under the current parameters (storage
// precision; the three stage pressures FP64).
fs_status tape_bind(fs_ctx* c, Tape* tp) {
  const size_t cb = c->Lc.total * c->S();
  const size_t fb[3] = {c->Lu.total * c->S(), c->Lv.total * c->S(), c->Lw.total * c->S()};
  const int n = c->prm.reinit_iterations;
  const size_t ncell = 4 + 3 * (size_t)n, nface = 27;
  while (c->tape_cells.size() < ncell) {
    void* p = nullptr;
    CKS(dalloc(c, &p, cb));
    c->tape_cells.push_back(p);
  }
  while (c->tape_faces.size() < nface) {
    void* p = nullptr;
    CKS(dalloc(c, &p, fb[c->tape_faces.size() % 3]));
    c->tape_faces.push_back(p);
  }
  while (c->tape_p.size() < 3) {
    double* p = nullptr;
    CKS(dalloc(c, (void**)&p, c->Lc.total * sizeof(double)));
    c->tape_p.push_back(p);
  }
  size_t q = 0;
  for (int m = 0; m < 4; ++m) tp->ls[m] = c->tape_cells[q++];
  for (int m = 0; m < 3; ++m) tp->p[m] = c->tape_p[m];
  for (int b = 0; b < 3; ++b) {
    tp->re[b].resize(n);
    for (int it = 0; it < n; ++it) tp->re[b][it] = c->tape_cells[q++];
  }
  size_t f = 0;
  for (int st = 0; st < 3; ++st)
    for (int k = 0; k < 3; ++k)
      for (int a = 0; a < 3; ++a) tp->vel[st][k][a] = c->tape_faces[f++];
  return FS_OK;
}

fs_status zero_cell(fs_ctx* c, double* p) {
  CK(cudaMemsetAsync(p, 0, c->Lc.total * sizeof(double), c->stream));
  return FS_OK;
}
fs_status zero_faces(fs_ctx* c, double* const t[3]) {
  const Lay* lays[3] = {&c->Lu, &c->Lv, &c->Lw};
  for (int a = 0; a < 3; ++a) CK(cudaMemsetAsync(t[a], 0, lays[a]->total * sizeof(double), c->stream));
  return FS_OK;
}
fs_status copy_cell(fs_ctx* c, double* dst, const double* src) {
  CK(cudaMemcpyAsync(dst, src, c->Lc.total * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  return FS_OK;
}
// copy three face fields of the storage precision (primal states)
fs_status copy_fields(fs_ctx* c, void* const dst[3], void* const src[3]) {
  const Lay* lays[3] = {&c->Lu, &c->Lv, &c->Lw};
  for (int a = 0; a < 3; ++a)
    CK(cudaMemcpyAsync(dst[a], src[a], lays[a]->total * c->S(), cudaMemcpyDeviceToDevice, c->stream));
  return FS_OK;
}
fs_status copy_faces(fs_ctx* c, double* const dst[3], double* const src[3]) {
  const Lay* lays[3] = {&c->Lu, &c->Lv, &c->Lw};
  for (int a = 0; a < 3; ++a)
    CK(cudaMemcpyAsync(dst[a], src[a], lays[a]->total * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  return FS_OK;
}
void axpy_faces(fs_ctx* c, double* const out[3], double* const x[3], double a) {
  const Lay* lays[3] = {&c->Lu, &c->Lv, &c->Lw};
  for (int q = 0; q < 3; ++q) adj_axpy(out[q], x[q], a, *lays[q], c->stream);
  c->launches += 3;
}

// One forward-Euler WENO5 level-set update fe = src - dt L(src; vel): given
// out_bar (bar of c1 * fe), src_bar = its bar w.r.t. src (overwritten) and
// vel_bar += its bar w.r.t. the velocity.  src is refilled in its ghosts.
template <class S>
fs_status adj_levelset_fe(fs_ctx* c, void* src, void* const vel[3], const double* out_bar, double c1,
                          double* src_bar, double* const vel_bar[3], double dt) {
  CKS(zero_cell(c, src_bar));
  fill_extrap<S>(F<S>(src), c->Lc, c->stream);
  adj_weno_levelset<S>(F<S>(src), F<S>(vel[0]), F<S>(vel[1]), F<S>(vel[2]), out_bar, src_bar, vel_bar[0], vel_bar[1], vel_bar[2], c->Lc, c->Lu,
                    c->Lv, c->Lw, c->grid.dx, c->prm.weno_epsilon, dt, c1, c->stream);
  adj_extrap(src_bar, c->Lc, c->stream);
  c->launches += 3;
  CK(cudaGetLastError());
  return FS_OK;
}

// One reinitialisation block B (S from its input, n Sussman steps) given the
// inputs of its pseudo-steps: x_bar (overwritten) = B'^T z_bar.
template <class S>
fs_status adj_reinit_block(fs_ctx* c, const std::vector<void*>& ys, const double* z_bar, double* x_bar) {
  const fs_params& P = c->prm;
  const int n = (int)ys.size();
  if (n == 0) return copy_cell(c, x_bar, z_bar);
  const double dx = c->grid.dx, dtau = dx / P.reinit_scaling;
  double *A = c->awork_c[2], *B = c->awork_c[3], *sbar = c->awork_c[4];
  sign_function<S>(F<S>(ys[0]), F<S>(c->sgn), c->Lc, dx, c->stream);
  CKS(zero_cell(c, sbar));
  CKS(copy_cell(c, A, z_bar));
  for (int it = n - 1; it >= 0; --it) {
    CKS(zero_cell(c, B));
    fill_extrap<S>(F<S>(ys[it]), c->Lc, c->stream);
    adj_sussman<S>(F<S>(ys[it]), F<S>(c->sgn), A, B, sbar, c->Lc, dx, P.weno_epsilon, dtau, 1.0,
                (P.flags & FS_FLAG_REINIT_TYPO) ? 1 : 0, c->stream);
    adj_extrap(B, c->Lc, c->stream);
    std::swap(A, B);
  }
  adj_sign<S>(F<S>(ys[0]), sbar, A, c->Lc, dx, c->stream);
  c->launches += 2 + 3 * n;
  CKS(copy_cell(c, x_bar, A));
  CK(cudaGetLastError());
  return FS_OK;
}

// Projection with the RK combination out = c0 base + c1 val: given out_bar,
// in_bar (overwritten) = bar of u*, base_bar += c0 out_bar (when base_bar),
// phi_bar and the density bars accumulate.  ustar, p: the forward's input
// velocity and pressure; phi the level set it used.
template <class S>
fs_status adj_projection(fs_ctx* c, void* phi, void* const ustar[3], const double* p, double* const out_bar[3],
                         double c1, double* const in_bar[3], double* phi_bar, double dt) {
  const fs_params& P = c->prm;
  const double dx = c->grid.dx;
  cudaStream_t s = c->stream;
  (void)ustar;  // the map is affine in u*: its derivative does not depend on it
  double *pbar = c->awork_c[0], *lam = c->awork_c[1];
  CKS(zero_cell(c, pbar));
  CKS(zero_cell(c, lam));
  const Lay* lays[3] = {&c->Lu, &c->Lv, &c->Lw};
  for (int a = 0; a < 3; ++a)
    adj_velcorr<S>(p, F<S>(phi), out_bar[a], in_bar[a], pbar, phi_bar, c->a_rho, *lays[a], c->Lc, a, dx, dt,
                   P.rho_neg, P.rho_pos, c1, s);
  c->launches += 5;
  CK(cudaGetLastError());
  // lambda = A^-1 p_bar (A symmetric): the second solve with the same
  // operator, to the forward's tolerance relative to its own right-hand
  // side, in the forward's arithmetic: FP64 PCG in FP64 contexts, the FP32
  // solve with FP64 defect correction in FP32 contexts
  int it = 0, st = 0;
  double rel = 0.0;
  if constexpr (sizeof(S) == sizeof(float)) {
    int outer = 0;
    CKS(mixed_solve<S>(c, F<S>(phi), pbar, lam, &it, &outer, &rel, &st));
  } else {
    build_pressure_operator<S, double>(F<S>(phi), c->Lc, dx, P.rho_neg, P.rho_pos, c->a_ax, c->a_ay, c->a_az,
                                       c->a_diag, c->scalars + 12, deflate(c), s);
    Op7<double> A{c->a_ax, c->a_ay, c->a_az, c->a_diag, c->Lc, 1, c->scalars + 12};
    CKS(run_pcg<double>(c, 3, A, pbar, lam, c->a_r, c->a_p, c->a_q, P.tolerance, std::max(P.max_iteration, 1),
                        FS_STOP_RELATIVE, &it, &rel, &st));
  }
  if (st != PCG_CONVERGED) {
    c->adj_unconverged += 1;
    c->adj_worst_rel = std::max(c->adj_worst_rel, rel);
    std::snprintf(c->adj_note, sizeof c->adj_note, "pressure: status %d after %d iterations, residual %.3e", st, it,
                  rel);
  }
  adj_sum(lam, c->Lc, c->partials, c->tickets + 4, c->scalars + 14, s);
  for (int a = 0; a < 3; ++a) adj_divergence(lam, c->scalars + 14, in_bar[a], *lays[a], c->Lc, a, dx, dt, s);
  adj_pressure_operator<S>(F<S>(phi), lam, p, phi_bar, c->a_rho, c->Lc, dx, P.rho_neg, P.rho_pos, deflate(c), s);
  c->launches += 5;
  CK(cudaGetLastError());
  return FS_OK;
}

// Semi-implicit viscosity x = M(phi)^-1 r(ug, phi): given out_bar (wall rows
// cleared here), in_bar (overwritten) = bar of ug; phi and density bars
// accumulate.  ug, x: the forward's input and output velocities.
template <class S>
fs_status adj_viscosity(fs_ctx* c, void* phi, void* const ug[3], void* const x[3], double* const out_bar[3],
                        double* const in_bar[3], double* phi_bar, double dt) {
  const fs_params& P = c->prm;
  const double dx = c->grid.dx;
  cudaStream_t s = c->stream;
  const Lay* lays[3] = {&c->Lu, &c->Lv, &c->Lw};
  CKS(zero_faces(c, in_bar));
  const bool shared = c->a_vs[1][0] == c->a_vs[0][0];
  for (int a = 0; a < 3; ++a) {
    if (shared) {
      // FP32 contexts share one FP64 system for the three components, whose
      // face layouts differ: clear it, so that the ghost entries the
      // matrix-free CG reads (couplings and vector values beyond the
      // component's interior) are zero again and not the previous
      // component's interior values
      const size_t fmax = std::max(c->Lu.total, std::max(c->Lv.total, c->Lw.total)) * sizeof(double);
      for (int m = 0; m < 9; ++m) CK(cudaMemsetAsync(c->a_vs[a][m], 0, fmax, s));
    }
    viscosity_system<S, double>(F<S>(phi), F<S>(ug[0]), F<S>(ug[1]), F<S>(ug[2]), c->Lc, c->Lu, c->Lv, c->Lw, a, dx,
                                dt, P.rho_neg, P.rho_pos, P.mu_neg, P.mu_pos, c->a_vs[a][0], c->a_vs[a][1],
                                c->a_vs[a][2], c->a_vs[a][3], c->a_vs[a][4], s);
    CK(cudaMemcpyAsync(c->a_vxb[a], out_bar[a], lays[a]->total * sizeof(double), cudaMemcpyDeviceToDevice, s));
    adj_zero_walls(c->a_vxb[a], *lays[a], a, s);  // wall rows are the constant zero
    CK(cudaMemsetAsync(c->a_vlam[a], 0, lays[a]->total * sizeof(double), s));
    Op7<double> A{c->a_vs[a][0], c->a_vs[a][1], c->a_vs[a][2], c->a_vs[a][3], *lays[a]};
    int it = 0, st = 0;
    CKS(run_pcg<double>(c, 120 + a, A, c->a_vxb[a], c->a_vlam[a], c->a_vs[a][6], c->a_vs[a][7], c->a_vs[a][8],
                        P.viscosity_tolerance, std::max(P.viscosity_max_iteration, 1), FS_STOP_RELATIVE, &it, nullptr,
                        &st));
    if (st != PCG_CONVERGED) {
      c->adj_unconverged += 1;
      std::snprintf(c->adj_note, sizeof c->adj_note, "viscosity component %d: status %d after %d iterations", a, st, it);
    }
    adj_visc<S>(F<S>(phi), F<S>(ug[0]), F<S>(ug[1]), F<S>(ug[2]), F<S>(x[a]), c->a_vlam[a], in_bar[0], in_bar[1],
                in_bar[2], phi_bar, c->a_rho, c->Lc, c->Lu, c->Lv, c->Lw, a, dx, dt, P.rho_neg, P.rho_pos, P.mu_neg,
                P.mu_pos, s);
    c->launches += 3;
  }
  CK(cudaGetLastError());
  return FS_OK;
}

// WENO5 self-advection of u, v, w: in_bar (overwritten) from out_bar.
template <class S>
fs_status adj_velocity_advect(fs_ctx* c, void* const uin[3], double* const out_bar[3], double* const in_bar[3],
                              double dt) {
  CKS(zero_faces(c, in_bar));
  const Lay* lays[3] = {&c->Lu, &c->Lv, &c->Lw};
  for (int a = 0; a < 3; ++a)
    adj_weno_mac<S>(F<S>(uin[a]), F<S>(uin[0]), F<S>(uin[1]), F<S>(uin[2]), out_bar[a], in_bar[a], in_bar[0], in_bar[1], in_bar[2], *lays[a],
                 c->Lu, c->Lv, c->Lw, a, c->grid.dx, velocity_epsilon(c), dt, c->stream);
  c->launches += 3;
  CK(cudaGetLastError());
  return FS_OK;
}

fs_status adj_check(fs_ctx* c) {
  if (c->prm.surface_tension != 0.0) {
    set_error("adjoints do not cover the surface-tension jump terms");
    return FS_NOT_SUPPORTED;
  }
  if (c->prm.velocity_scheme != FS_VELOCITY_WENO5) {
    set_error("adjoints cover the WENO5 velocity advection only");
    return FS_NOT_SUPPORTED;
  }
  if (c->prm.fast_sweeping) {
    set_error("adjoints cover the Sussman reinitialisation only");
    return FS_NOT_SUPPORTED;
  }
  if (c->prm.flags & FS_FLAG_FAITHFUL_PROJECTION) {
    set_error("adjoints follow the corrected projection only");
    return FS_NOT_SUPPORTED;
  }
  if (c->prm.viscosity == 2) {
    set_error("adjoints cover the semi-implicit viscosity only");
    return FS_NOT_SUPPORTED;
  }
  return adj_alloc(c);
}

// The whole step: forward recomputed with a tape from the current state,
// then the reverse sweep.  On entry abar holds the bars of the step's
// output; on return the bars of its input (phi, u, v, w) and a_rho has the
// density bars added.  The fields end in the step's output state.
template <class S>
fs_status step_adjoint_t(fs_ctx* c, double dt, fs_step_report* rep) {
  const fs_params& P = c->prm;
  Tape tp;
  CKS(tape_bind(c, &tp));
  void* u0[3];
  for (int a = 0; a < 3; ++a) u0[a] = tp.vel[0][0][a];  // the step's initial velocity (first stage input)
  fs_status fw = step_t<S>(c, dt, rep, &tp);
  if (fw != FS_OK && fw != FS_NOT_CONVERGED) return fw;
  const int order = P.order;
  // ---- reinitialisation blocks
  void* phiA = tp.ls[3];
  double *phibar = c->abar[0], *phiAbar = c->awork_c[5];
  CKS(zero_cell(c, phiAbar));
  {
    double *zb = c->awork_c[0], *xb = c->awork_c[1];  // free here: the projection adjoint runs later
    const int nb = order == 3 ? 3 : 2;
    const double c0s[3] = {0.0, order == 3 ? 0.75 : 0.5, 1.0 / 3.0};
    const double c1s[3] = {1.0, order == 3 ? 0.25 : 0.5, 2.0 / 3.0};
    // bar of the last block's output is phibar; walk the blocks backwards
    CKS(copy_cell(c, zb, phibar));
    for (int b = nb - 1; b >= 0; --b) {
      adj_axpy(phiAbar, zb, c0s[b], c->Lc, c->stream);  // base term
      CK(cudaMemsetAsync(xb, 0, c->Lc.total * sizeof(double), c->stream));
      // the block's own output is scaled by c1
      adj_axpy(xb, zb, c1s[b], c->Lc, c->stream);
      CKS(adj_reinit_block<S>(c, tp.re[b], xb, zb));  // zb <- bar of the block input
      c->launches += 2;
    }
    adj_axpy(phiAbar, zb, 1.0, c->Lc, c->stream);  // the first block's input is phiA
    c->launches += 1;
  }
  // ---- velocity stages, backwards
  const int ns = order;
  const double vc0[3] = {0.0, order == 3 ? 0.75 : 0.5, 1.0 / 3.0};
  const double vc1[3] = {1.0, order == 3 ? 0.25 : 0.5, 2.0 / 3.0};
  double* const* ubar = &c->abar[1];
  double* cur[3];   // bar of the current stage's output
  double* u0bar[3];
  for (int a = 0; a < 3; ++a) { cur[a] = c->awork_f[0][a]; u0bar[a] = c->awork_f[3][a]; }
  CKS(copy_faces(c, cur, ubar));
  CKS(zero_faces(c, u0bar));
  for (int st = ns - 1; st >= 0; --st) {
    if (vc0[st] != 0.0) axpy_faces(c, u0bar, cur, vc0[st]);
    double* pin[3] = {c->awork_f[1][0], c->awork_f[1][1], c->awork_f[1][2]};
    CKS(adj_projection<S>(c, phiA, tp.vel[st][2], tp.p[st], cur, vc1[st], pin, phiAbar, dt));
    double* gin[3] = {c->awork_f[2][0], c->awork_f[2][1], c->awork_f[2][2]};
    if (P.viscosity) {
      CKS(adj_viscosity<S>(c, phiA, tp.vel[st][1], tp.vel[st][2], pin, gin, phiAbar, dt));
    } else {
      CKS(copy_faces(c, gin, pin));
    }
    // gravity adds a constant; the no-penetration zeroing clears the wall bars
    const Lay* lays[3] = {&c->Lu, &c->Lv, &c->Lw};
    for (int a = 0; a < 3; ++a) adj_zero_walls(gin[a], *lays[a], a, c->stream);
    c->launches += 3;
    CKS(adj_velocity_advect<S>(c, tp.vel[st][0], gin, cur, dt));  // cur <- bar of the stage input
  }
  axpy_faces(c, u0bar, cur, 1.0);  // the first stage's input is u0
  // ---- level set: phiA from phi0 with the initial velocity u0
  double* b1 = c->awork_c[0];
  double* b2 = c->awork_c[1];
  CKS(zero_cell(c, phibar));
  void* const* u0p = u0;
  if (order == 3 && !(P.flags & FS_FLAG_LEVELSET_FORWARD_EULER)) {
    // phiA = 1/3 phi0 + 2/3 FE(phi2); phi2 = 3/4 phi0 + 1/4 FE(phi1); phi1 = FE(phi0)
    adj_axpy(phibar, phiAbar, 1.0 / 3.0, c->Lc, c->stream);
    CKS(adj_levelset_fe<S>(c, tp.ls[2], u0p, phiAbar, 2.0 / 3.0, b2, u0bar, dt));  // b2 = bar of phi2
    adj_axpy(phibar, b2, 0.75, c->Lc, c->stream);
    CKS(adj_levelset_fe<S>(c, tp.ls[1], u0p, b2, 0.25, b1, u0bar, dt));            // b1 = bar of phi1
    CKS(adj_levelset_fe<S>(c, tp.ls[0], u0p, b1, 1.0, b2, u0bar, dt));             // b2 = bar of phi0 via FE
    adj_axpy(phibar, b2, 1.0, c->Lc, c->stream);
    c->launches += 3;
  } else if (order == 3) {
    CKS(adj_levelset_fe<S>(c, tp.ls[0], u0p, phiAbar, 1.0, b2, u0bar, dt));
    adj_axpy(phibar, b2, 1.0, c->Lc, c->stream);
    c->launches += 1;
  } else {
    // Heun: phiA = 1/2 phi0 + 1/2 FE(phi1), phi1 = FE(phi0)
    adj_axpy(phibar, phiAbar, 0.5, c->Lc, c->stream);
    CKS(adj_levelset_fe<S>(c, tp.ls[1], u0p, phiAbar, 0.5, b1, u0bar, dt));
    CKS(adj_levelset_fe<S>(c, tp.ls[0], u0p, b1, 1.0, b2, u0bar, dt));
    adj_axpy(phibar, b2, 1.0, c->Lc, c->stream);
    c->launches += 2;
  }
  CKS(copy_faces(c, ubar, u0bar));
  CK(cudaGetLastError());
  return fw;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

void fs_params_default(fs_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof *p);
  p->rho_neg = 1000.0;
  p->rho_pos = 1.0;
  p->mu_neg = 1e-3;
  p->mu_pos = 1.8e-5;
  p->gravity[0] = 0.0;
  p->gravity[1] = -9.8;
  p->gravity[2] = 0.0;
  p->weno_epsilon = 1e-6;
  p->reinit_iterations = 10;
  p->reinit_scaling = 5;
  p->order = 3;
  p->precision = FS_PRECISION_FP64;
  p->stop = FS_STOP_RELATIVE;
  p->tolerance = 1e-6;
  p->max_iteration = 20000;
  p->inner_tolerance = 1e-3;
  p->max_outer = 20;
  p->viscosity = 1;
  p->viscosity_tolerance = 1e-8;
  p->viscosity_max_iteration = 1000;
  p->cfl = 0.5;
  p->flags = 0;
  p->pressure_preconditioner = FS_PRECOND_DEFAULT;
  p->reliable_delta = 0.1;
  p->flux_arithmetic = 2;
  p->verbose = 0;
  p->host_loop = 0;
}

const char* fs_status_str(fs_status s) {
  switch (s) {
    case FS_OK: return "ok";
    case FS_INVALID_ARG: return "invalid argument";
    case FS_OOM: return "out of device memory";
    case FS_NOT_CONVERGED: return "iterative solve not converged";
    case FS_NONFINITE: return "non-finite value";
    case FS_CUDA_ERROR: return "CUDA error";
    case FS_TIMEOUT: return "timeout";
    case FS_NOT_SUPPORTED: return "not supported";
  }
  return "unknown status";
}

const char* fs_last_error(void) { return g_last_error; }

fs_status fs_create(const fs_grid_desc* grid, const fs_params* params, fs_ctx** out) {
  if (!grid || !out) { set_error("NULL argument"); return FS_INVALID_ARG; }
  *out = nullptr;
  if (grid->nx < 3 || grid->ny < 3 || grid->nz < 3 || !(grid->dx > 0)) {
    set_error("grid must be at least 3^3 cells with dx > 0");
    return FS_INVALID_ARG;
  }
  const int64_t cells = (int64_t)grid->nx * grid->ny * grid->nz;
  if (grid->nx > 4096 || grid->ny > 4096 || grid->nz > 4096 || cells > (int64_t)1 << 32) {
    set_error("grid too large for one context");
    return FS_INVALID_ARG;
  }
  fs_params prm;
  if (params) prm = *params; else fs_params_default(&prm);
  CKS(check_params(&prm));
  fs_ctx* c = new (std::nothrow) fs_ctx();
  if (!c) { set_error("host allocation failed"); return FS_OOM; }
  c->grid = *grid;
  c->prm = prm;
  c->fp32 = prm.precision == FS_PRECISION_FP32_REFINE;
  apply_params(c);
  if (fs_status ps = setup_pipe(c); ps != FS_OK) {
    delete c;
    return ps;
  }
  c->Lc = make_lay(grid->nx, grid->ny, grid->nz);
  c->Lu = make_lay(grid->nx + 1, grid->ny, grid->nz);
  c->Lv = make_lay(grid->nx, grid->ny + 1, grid->nz);
  c->Lw = make_lay(grid->nx, grid->ny, grid->nz + 1);
  auto fail = [&](fs_status s) { release(c); delete c; return s; };
  if (cudaGetDevice(&c->device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      cudaEventCreate(&c->evp0) != cudaSuccess || cudaEventCreate(&c->evp1) != cudaSuccess) {
    set_error("CUDA stream/event creation failed: %s", cudaGetErrorString(cudaGetLastError()));
    return fail(FS_CUDA_ERROR);
  }
  const size_t S = c->S();
  const size_t cb = c->Lc.total * S, ub = c->Lu.total * S, vb = c->Lv.total * S, wb = c->Lw.total * S;
  const size_t c8 = c->Lc.total * sizeof(double);
  const size_t V = c->fp32 ? sizeof(float) : sizeof(double);
  const size_t cv = c->Lc.total * V;
  fs_status s = FS_OK;
  void** cell_s[] = {&c->phi, &c->s1, &c->s2, &c->s3, &c->s4, &c->sgn};
  for (void** p : cell_s) if ((s = dalloc(c, p, cb)) != FS_OK) return fail(s);
  void** fu[] = {&c->u, &c->u0, &c->ua};
  void** fv[] = {&c->v, &c->v0, &c->va};
  void** fw[] = {&c->w, &c->w0, &c->wa};
  for (void** p : fu) if ((s = dalloc(c, p, ub)) != FS_OK) return fail(s);
  for (void** p : fv) if ((s = dalloc(c, p, vb)) != FS_OK) return fail(s);
  for (void** p : fw) if ((s = dalloc(c, p, wb)) != FS_OK) return fail(s);
  double** d8[] = {&c->p64, &c->b64, &c->div64, &c->kappa};
  for (double** p : d8) if ((s = dalloc(c, (void**)p, c8)) != FS_OK) return fail(s);
  if ((s = dalloc(c, (void**)&c->fsfixed, c->Lc.total)) != FS_OK) return fail(s);
  if ((s = dalloc(c, (void**)&c->fsflag, sizeof(int))) != FS_OK) return fail(s);
  if (c->fp32 && (s = dalloc(c, (void**)&c->p64bak, c8)) != FS_OK) return fail(s);
  void** pv[] = {&c->pax, &c->pay, &c->paz, &c->pdiag, &c->pr, &c->pp, &c->pq};
  for (void** p : pv) if ((s = dalloc(c, p, cv)) != FS_OK) return fail(s);
  if (c->fp32) {
    if ((s = dalloc(c, &c->px, cv)) != FS_OK) return fail(s);
    if ((s = dalloc(c, &c->prhs, cv)) != FS_OK) return fail(s);
    if ((s = dalloc(c, (void**)&c->pdinv, c->Lc.total * sizeof(unsigned short))) != FS_OK) return fail(s);
    c->Lh = make_half_lay(c->Lc);
    const size_t hb = c->Lh.total;
    if ((s = dalloc(c, (void**)&c->rb_x, hb * sizeof(double))) != FS_OK) return fail(s);
    float** hv[] = {&c->rb_r, &c->rb_p, &c->rb_q, &c->rb_tau};
    for (float** p : hv) if ((s = dalloc(c, (void**)p, hb * sizeof(float))) != FS_OK) return fail(s);
    if ((s = dalloc(c, (void**)&c->rb_dinv, hb * sizeof(unsigned short))) != FS_OK) return fail(s);
  }
  if (prm.pipe) {
    const size_t fb[3] = {ub, vb, wb};
    for (int a = 0; a < 3; ++a)
      for (void** p : {&c->pgen[a], &c->pgx[a], &c->pgz[a]})
        if ((s = dalloc(c, p, fb[a])) != FS_OK) return fail(s);
  }
  if (prm.viscosity == 1) {
    const size_t fb[3] = {ub, vb, wb};
    for (int a = 0; a < 3; ++a)
      for (int m = 0; m < 9; ++m)
        if ((s = dalloc(c, &c->vs[a][m], fb[a])) != FS_OK) return fail(s);
  }
  // grid sizes of the Krylov kernels (occupancy queries; never under capture)
  cg_prepare<double, double>();
  cg_prepare<float, double>();
  cg_prepare<float, float>();
  int nblk = std::max(pcg_blocks(c->Lu), std::max(pcg_blocks(c->Lv), pcg_blocks(c->Lw))) * 2 + 64;
  for (const Lay* L : {&c->Lc, &c->Lu, &c->Lv, &c->Lw}) nblk = std::max(nblk, cg_max_blocks(*L));
  if (c->fp32) nblk = std::max(nblk, rb_blocks(c->Lh));
  if ((s = dalloc(c, (void**)&c->partials, (size_t)nblk * 3 * sizeof(double))) != FS_OK) return fail(s);
  if ((s = dalloc(c, (void**)&c->tickets, 8 * sizeof(unsigned int))) != FS_OK) return fail(s);
  if ((s = dalloc(c, (void**)&c->scalars, 16 * sizeof(double))) != FS_OK) return fail(s);
  if ((s = dalloc(c, (void**)&c->st, sizeof(PcgState))) != FS_OK) return fail(s);
  const int64_t maxf = std::max(std::max(c->Lu.total, c->Lv.total), std::max(c->Lw.total, c->Lc.total));
  if ((s = dalloc(c, (void**)&c->staging, (size_t)maxf * sizeof(double))) != FS_OK) return fail(s);
  if (cudaMallocHost((void**)&c->st_host, sizeof(PcgState)) != cudaSuccess ||
      cudaMallocHost((void**)&c->sc_host, 16 * sizeof(double)) != cudaSuccess) {
    set_error("pinned host allocation failed");
    return fail(FS_OOM);
  }
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    set_error("initialisation failed: %s", cudaGetErrorString(cudaGetLastError()));
    return fail(FS_CUDA_ERROR);
  }
  *out = c;
  return FS_OK;
}

fs_status fs_destroy(fs_ctx* c) {
  if (!c) return FS_OK;
  cudaStreamSynchronize(c->stream);
  release(c);
  delete c;
  return FS_OK;
}

fs_status fs_set_params(fs_ctx* c, const fs_params* p) {
  if (!c || !p) { set_error("NULL argument"); return FS_INVALID_ARG; }
  CKS(check_params(p));
  if (p->precision != c->prm.precision) { set_error("precision is fixed at creation"); return FS_INVALID_ARG; }
  if ((p->pipe != 0) != (c->prm.pipe != 0)) { set_error("the pipe mode is fixed at creation"); return FS_INVALID_ARG; }
  if (p->viscosity == 1 && !c->vs[0][0]) {
    set_error("semi-implicit viscosity buffers were not allocated at creation");
    return FS_INVALID_ARG;
  }
  const fs_params old = c->prm;
  c->prm = *p;
  if (fs_status ps = setup_pipe(c); ps != FS_OK) {
    c->prm = old;
    setup_pipe(c);
    return ps;
  }
  apply_params(c);
  // captured solver graphs hold the operator's arithmetic and preconditioner
  // as kernel arguments: capture them again under the new settings
  for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);
  c->graphs.clear();
  return FS_OK;
}

fs_status fs_memory_bytes(const fs_ctx* c, int64_t* bytes) {
  if (!c || !bytes) { set_error("NULL argument"); return FS_INVALID_ARG; }
  *bytes = c->bytes;
  return FS_OK;
}

static void** field_ptr(fs_ctx* c, int field) {
  switch (field) {
    case FS_FIELD_PHI: return &c->phi;
    case FS_FIELD_U: return &c->u;
    case FS_FIELD_V: return &c->v;
    case FS_FIELD_W: return &c->w;
    default: return nullptr;
  }
}

static fs_status upload_from_staging(fs_ctx* c, int field) {
  const Lay& L = lay_of(c, field);
  if (is_adjoint_field(field)) {
    unpack_from_double<double>(c->abar[field - FS_FIELD_ADJ_PHI], c->staging, L, c->stream);
  } else if (field == FS_FIELD_PRESSURE) {
    unpack_from_double<double>(c->p64, c->staging, L, c->stream);
  } else {
    void* dst = *field_ptr(c, field);
    if (c->fp32) unpack_from_double<float>((float*)dst, c->staging, L, c->stream);
    else unpack_from_double<double>((double*)dst, c->staging, L, c->stream);
  }
  CK(cudaGetLastError());
  return FS_OK;
}

static fs_status download_to_staging(fs_ctx* c, int field) {
  const Lay& L = lay_of(c, field);
  if (is_adjoint_field(field)) pack_to_double<double>(c->staging, c->abar[field - FS_FIELD_ADJ_PHI], L, c->stream);
  else if (field == FS_FIELD_CURVATURE) pack_to_double<double>(c->staging, c->kappa, L, c->stream);
  else if (field == FS_FIELD_PRESSURE) pack_to_double<double>(c->staging, c->p64, L, c->stream);
  else if (field == FS_FIELD_DIVERGENCE) pack_to_double<double>(c->staging, c->div64, L, c->stream);
  else {
    void* src = *field_ptr(c, field);
    if (c->fp32) pack_to_double<float>(c->staging, (const float*)src, L, c->stream);
    else pack_to_double<double>(c->staging, (const double*)src, L, c->stream);
  }
  CK(cudaGetLastError());
  return FS_OK;
}

static int64_t field_count(const fs_ctx* c, int field) {
  const Lay& L = lay_of(c, field);
  return (int64_t)L.nx * L.ny * L.nz;
}

// fields accepted by upload (0..4 and the adjoint fields) and download (0..5 and the adjoint fields)
static fs_status check_field(fs_ctx* c, int field, bool upload) {
  if (is_adjoint_field(field)) return adj_check(c);
  if (field == FS_FIELD_CURVATURE && !upload) return FS_OK;
  if (field < FS_FIELD_PHI || field > (upload ? FS_FIELD_PRESSURE : FS_FIELD_DIVERGENCE)) {
    set_error("field %d cannot be %s", field, upload ? "uploaded" : "downloaded");
    return FS_INVALID_ARG;
  }
  return FS_OK;
}

fs_status fs_upload(fs_ctx* c, int field, const double* host, const int64_t* strides) {
  if (!c || !host) { set_error("NULL argument"); return FS_INVALID_ARG; }
  CKS(check_field(c, field, true));
  const Lay& L = lay_of(c, field);
  const int64_t n = field_count(c, field);
  if (strides) {
    std::vector<double> tmp((size_t)n);
    for (int k = 0; k < L.nz; ++k)
      for (int j = 0; j < L.ny; ++j)
        for (int i = 0; i < L.nx; ++i)
          tmp[((size_t)k * L.ny + j) * L.nx + i] = host[i * strides[0] + j * strides[1] + k * strides[2]];
    CK(cudaMemcpyAsync(c->staging, tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CKS(upload_from_staging(c, field));
    CK(cudaStreamSynchronize(c->stream));
    return FS_OK;
  }
  CK(cudaMemcpyAsync(c->staging, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CKS(upload_from_staging(c, field));
  CK(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_download(fs_ctx* c, int field, double* host, const int64_t* strides) {
  if (!c || !host) { set_error("NULL argument"); return FS_INVALID_ARG; }
  CKS(check_field(c, field, false));
  const Lay& L = lay_of(c, field);
  const int64_t n = field_count(c, field);
  CKS(download_to_staging(c, field));
  if (strides) {
    std::vector<double> tmp((size_t)n);
    CK(cudaMemcpyAsync(tmp.data(), c->staging, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int k = 0; k < L.nz; ++k)
      for (int j = 0; j < L.ny; ++j)
        for (int i = 0; i < L.nx; ++i)
          host[i * strides[0] + j * strides[1] + k * strides[2]] = tmp[((size_t)k * L.ny + j) * L.nx + i];
    return FS_OK;
  }
  CK(cudaMemcpyAsync(host, c->staging, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_upload_device(fs_ctx* c, int field, const double* dev) {
  if (!c || !dev) { set_error("NULL argument"); return FS_INVALID_ARG; }
  CKS(check_field(c, field, true));
  const Lay& L = lay_of(c, field);
  if (is_adjoint_field(field)) unpack_from_double<double>(c->abar[field - FS_FIELD_ADJ_PHI], dev, L, c->stream);
  else if (field == FS_FIELD_PRESSURE) unpack_from_double<double>(c->p64, dev, L, c->stream);
  else if (c->fp32) unpack_from_double<float>((float*)*field_ptr(c, field), dev, L, c->stream);
  else unpack_from_double<double>((double*)*field_ptr(c, field), dev, L, c->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_download_device(fs_ctx* c, int field, double* dev) {
  if (!c || !dev) { set_error("NULL argument"); return FS_INVALID_ARG; }
  CKS(check_field(c, field, false));
  const Lay& L = lay_of(c, field);
  if (is_adjoint_field(field)) pack_to_double<double>(dev, c->abar[field - FS_FIELD_ADJ_PHI], L, c->stream);
  else if (field == FS_FIELD_CURVATURE) pack_to_double<double>(dev, c->kappa, L, c->stream);
  else if (field == FS_FIELD_PRESSURE) pack_to_double<double>(dev, c->p64, L, c->stream);
  else if (field == FS_FIELD_DIVERGENCE) pack_to_double<double>(dev, c->div64, L, c->stream);
  else if (c->fp32) pack_to_double<float>(dev, (const float*)*field_ptr(c, field), L, c->stream);
  else pack_to_double<double>(dev, (const double*)*field_ptr(c, field), L, c->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

#define DISPATCH(c, fn, ...) ((c)->fp32 ? fn<float>(__VA_ARGS__) : fn<double>(__VA_ARGS__))

static fs_status timed_begin(fs_ctx* c) {
  CK(cudaEventRecord(c->ev0, c->stream));
  return FS_OK;
}

static fs_status timed_end(fs_ctx* c, float* ms) {
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  if (ms) CK(cudaEventElapsedTime(ms, c->ev0, c->ev1));
  return FS_OK;
}

fs_status fs_step(fs_ctx* c, double dt, fs_step_report* rep) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  if (c->pipe.on && c->prm.viscosity != 0) {
    // the pipe's semi-implicit viscosity is not built: the step runs as the
    // reference's with is_sourcing_active = false
    set_error("fs_step in the pipe mode needs viscosity = 0 (the pipe's viscosity is not built)");
    return FS_NOT_SUPPORTED;
  }
  if (!(dt > 0) || !std::isfinite(dt)) { set_error("dt must be positive and finite"); return FS_INVALID_ARG; }
  fs_step_report local{};
  fs_step_report* r = rep ? rep : &local;
  *r = fs_step_report{};
  c->launches = 0;
  c->pcg_ms = 0.0f;
  c->pcg_launched_iterations = 0;
  CKS(timed_begin(c));
  fs_status s = DISPATCH(c, step_t, c, dt, r);
  if (s != FS_OK && s != FS_NOT_CONVERGED) return s;
  CKS(timed_end(c, &r->ms));
  r->pcg_ms = c->pcg_ms;
  r->pcg_launched_iterations = c->pcg_launched_iterations;
  r->kernel_launches = c->launches;
  return s;
}

fs_status fs_curvature(fs_ctx* c, double* kappa_max) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  CKS(box_only(c, "fs_curvature"));
  CKS(DISPATCH(c, curvature_t, c));
  CK(cudaMemcpyAsync(c->sc_host + 13, c->scalars + 13, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (kappa_max) *kappa_max = c->sc_host[13];
  return FS_OK;
}

fs_status fs_cfl_dt(fs_ctx* c, double* dt) {
  if (!c || !dt) { set_error("NULL argument"); return FS_INVALID_ARG; }
  return DISPATCH(c, cfl_t, c, dt);
}

fs_status fs_project(fs_ctx* c, double dt, fs_solve_report* rep) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  if (!(dt > 0) || !std::isfinite(dt)) { set_error("dt must be positive and finite"); return FS_INVALID_ARG; }
  fs_solve_report local{};
  fs_solve_report* r = rep ? rep : &local;
  CKS(timed_begin(c));
  fs_status s = DISPATCH(c, project_t, c, dt, 0.0, 1.0, r);
  if (s != FS_OK && s != FS_NOT_CONVERGED) return s;
  CKS(timed_end(c, &r->ms));
  return s;
}

fs_status fs_advect_levelset(fs_ctx* c, double dt) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  const int order = c->prm.order, flags = c->prm.flags;
  // a single forward-Euler update, whatever the time order
  c->prm.order = 3;
  c->prm.flags |= FS_FLAG_LEVELSET_FORWARD_EULER;
  fs_status s = DISPATCH(c, advect_levelset_t, c, dt);
  c->prm.order = order;
  c->prm.flags = flags;
  if (s != FS_OK) return s;
  CK(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_apply_gravity(fs_ctx* c, double dt) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  if (!(dt > 0) || !std::isfinite(dt)) { set_error("dt must be positive and finite"); return FS_INVALID_ARG; }
  CKS(DISPATCH(c, gravity_t, c, dt));
  CK(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_advect_velocity(fs_ctx* c, double dt) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  CKS(DISPATCH(c, advect_velocity_t, c, dt));
  CK(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_reinitialize(fs_ctx* c) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  // one block: S from the current phi, reinit_iterations pseudo-steps
  fs_status s = c->fp32 ? reinit_block_t<float>(c, c->phi, c->s1, c->phi, 0.0, 1.0, c->s2, c->s3)
                        : reinit_block_t<double>(c, c->phi, c->s1, c->phi, 0.0, 1.0, c->s2, c->s3);
  if (s != FS_OK) return s;
  if (c->prm.reinit_iterations > 0) std::swap(c->phi, c->s1);
  CK(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_fast_sweeping(fs_ctx* c, int direction, int pairs) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  CKS(box_only(c, "fs_fast_sweeping"));
  if (direction < -1 || direction > 3 || pairs < 1 || pairs > 4) {
    set_error("direction must be -1..3 and pairs 1..4");
    return FS_INVALID_ARG;
  }
  fs_status s = c->fp32 ? fast_sweeping_t<float>(c, c->phi, c->s1, direction, pairs)
                        : fast_sweeping_t<double>(c, c->phi, c->s1, direction, pairs);
  if (s != FS_OK) return s;
  std::swap(c->phi, c->s1);
  CK(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_surface(fs_ctx* c, int64_t* n_vertices, int64_t* n_triangles) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  const cudaError_t e = c->fp32 ? polygonize<float>(F<float>(c->phi), c->Lc, c->grid.dx, &c->mesh, c->stream)
                                : polygonize<double>(F<double>(c->phi), c->Lc, c->grid.dx, &c->mesh, c->stream);
  if (e == cudaErrorInvalidValue) {
    set_error("grid too large for the surface extraction's 32-bit vertex numbers");
    return FS_INVALID_ARG;
  }
  if (e == cudaErrorMemoryAllocation) {
    set_error("device memory for the surface mesh");
    return FS_OOM;
  }
  CK(e);
  c->launches += 9;
  if (n_vertices) *n_vertices = c->mesh.nv;
  if (n_triangles) *n_triangles = c->mesh.nt;
  return FS_OK;
}

fs_status fs_surface_download(fs_ctx* c, double* xyz, double* normals, int32_t* triangles) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  const SurfaceMesh& m = c->mesh;
  if (xyz && m.nv) CK(cudaMemcpy(xyz, m.xyz, m.nv * 3 * sizeof(double), cudaMemcpyDeviceToHost));
  if (normals && m.nv) CK(cudaMemcpy(normals, m.normals, m.nv * 3 * sizeof(double), cudaMemcpyDeviceToHost));
  if (triangles && m.nt) CK(cudaMemcpy(triangles, m.tri, m.nt * 3 * sizeof(int), cudaMemcpyDeviceToHost));
  return FS_OK;
}

fs_status fs_write_obj(fs_ctx* c, const char* path) {
  if (!c || !path) { set_error("NULL argument"); return FS_INVALID_ARG; }
  int64_t nv = 0, nt = 0;
  CKS(fs_surface(c, &nv, &nt));
  std::vector<double> xyz(3 * nv), nrm(3 * nv);
  std::vector<int32_t> tri(3 * nt);
  CKS(fs_surface_download(c, xyz.data(), nrm.data(), tri.data()));
  FILE* f = std::fopen(path, "w");
  if (!f) { set_error("cannot open %s", path); return FS_INVALID_ARG; }
  bool ok = true;
  for (int64_t v = 0; v < nv && ok; ++v)
    ok = std::fprintf(f, "v %.9g %.9g %.9g\n", xyz[3 * v], xyz[3 * v + 1], xyz[3 * v + 2]) > 0;
  for (int64_t v = 0; v < nv && ok; ++v)
    ok = std::fprintf(f, "vn %.9g %.9g %.9g\n", nrm[3 * v], nrm[3 * v + 1], nrm[3 * v + 2]) > 0;
  for (int64_t t = 0; t < nt && ok; ++t)
    ok = std::fprintf(f, "f %d//%d %d//%d %d//%d\n", tri[3 * t], tri[3 * t], tri[3 * t + 1], tri[3 * t + 1],
                      tri[3 * t + 2], tri[3 * t + 2]) > 0;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) { set_error("writing %s failed", path); return FS_INVALID_ARG; }
  return FS_OK;
}

fs_status fs_viscosity(fs_ctx* c, double dt, int* iterations) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  CKS(box_only(c, "fs_viscosity"));
  if (!(dt > 0)) { set_error("dt must be positive"); return FS_INVALID_ARG; }
  CKS(DISPATCH(c, viscosity_t, c, dt, iterations));
  CK(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

// ---- state I/O

// LEVELSET_3D::Write/Read (LEVELSET_3D.h:1132-1200): int32 i_start, j_start,
// k_start, i_res, j_res, k_res; float64 x_min, y_min, z_min, x_max, y_max,
// z_max; int32 ghost_width; then phi(i, j, k) as float64 with i fastest,
// k slowest.  No padding between the fields.
fs_status fs_write_levelset(fs_ctx* c, const char* path, const double* grid_min) {
  if (!c || !path) { set_error("NULL argument"); return FS_INVALID_ARG; }
  const int nx = c->grid.nx, ny = c->grid.ny, nz = c->grid.nz;
  std::vector<double> phi((size_t)nx * ny * nz);
  CKS(fs_download(c, FS_FIELD_PHI, phi.data(), nullptr));
  FILE* f = std::fopen(path, "wb");
  if (!f) { set_error("cannot open %s for writing", path); return FS_INVALID_ARG; }
  const int32_t hdr_i[6] = {0, 0, 0, nx, ny, nz};
  const double mn[3] = {grid_min ? grid_min[0] : 0.0, grid_min ? grid_min[1] : 0.0, grid_min ? grid_min[2] : 0.0};
  const double hdr_d[6] = {mn[0], mn[1], mn[2], mn[0] + (nx - 1) * c->grid.dx, mn[1] + (ny - 1) * c->grid.dx,
                           mn[2] + (nz - 1) * c->grid.dx};
  const int32_t ghost = GH;
  bool ok = std::fwrite(hdr_i, sizeof hdr_i, 1, f) == 1 && std::fwrite(hdr_d, sizeof hdr_d, 1, f) == 1 &&
            std::fwrite(&ghost, sizeof ghost, 1, f) == 1 &&
            std::fwrite(phi.data(), sizeof(double), phi.size(), f) == phi.size();
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) { set_error("short write to %s", path); return FS_INVALID_ARG; }
  return FS_OK;
}

fs_status fs_read_levelset(fs_ctx* c, const char* path, double* grid_min) {
  if (!c || !path) { set_error("NULL argument"); return FS_INVALID_ARG; }
  FILE* f = std::fopen(path, "rb");
  if (!f) { set_error("cannot open %s", path); return FS_INVALID_ARG; }
  int32_t hdr_i[6];
  double hdr_d[6];
  int32_t ghost = 0;
  bool ok = std::fread(hdr_i, sizeof hdr_i, 1, f) == 1 && std::fread(hdr_d, sizeof hdr_d, 1, f) == 1 &&
            std::fread(&ghost, sizeof ghost, 1, f) == 1;
  const int nx = c->grid.nx, ny = c->grid.ny, nz = c->grid.nz;
  if (ok && (hdr_i[3] != nx || hdr_i[4] != ny || hdr_i[5] != nz)) {
    std::fclose(f);
    set_error("%s holds a %d x %d x %d level set, the context is %d x %d x %d", path, hdr_i[3], hdr_i[4], hdr_i[5], nx,
              ny, nz);
    return FS_INVALID_ARG;
  }
  if (ok) {
    const double dx = (hdr_d[3] - hdr_d[0]) / (nx > 1 ? nx - 1 : 1);
    if (std::fabs(dx - c->grid.dx) > 1e-12 * c->grid.dx) {
      std::fclose(f);
      set_error("%s has grid spacing %.17g, the context %.17g", path, dx, c->grid.dx);
      return FS_INVALID_ARG;
    }
  }
  std::vector<double> phi((size_t)nx * ny * nz);
  ok = ok && std::fread(phi.data(), sizeof(double), phi.size(), f) == phi.size();
  std::fclose(f);
  if (!ok) { set_error("%s is truncated or not a level-set file", path); return FS_INVALID_ARG; }
  if (grid_min) {
    grid_min[0] = hdr_d[0];
    grid_min[1] = hdr_d[1];
    grid_min[2] = hdr_d[2];
  }
  return fs_upload(c, FS_FIELD_PHI, phi.data(), nullptr);
}

// Checkpoint of the step state: "FSB200ST", uint32 version 1, int32 nx, ny,
// nz, float64 dx, then phi, u, v, w, pressure as float64 interior values
// (x fastest), each field in the layout of fs_download.
static const char kStateMagic[8] = {'F', 'S', 'B', '2', '0', '0', 'S', 'T'};

fs_status fs_write_state(fs_ctx* c, const char* path) {
  if (!c || !path) { set_error("NULL argument"); return FS_INVALID_ARG; }
  FILE* f = std::fopen(path, "wb");
  if (!f) { set_error("cannot open %s for writing", path); return FS_INVALID_ARG; }
  const uint32_t version = 1;
  const int32_t dims[3] = {c->grid.nx, c->grid.ny, c->grid.nz};
  bool ok = std::fwrite(kStateMagic, 8, 1, f) == 1 && std::fwrite(&version, 4, 1, f) == 1 &&
            std::fwrite(dims, sizeof dims, 1, f) == 1 && std::fwrite(&c->grid.dx, 8, 1, f) == 1;
  const int fields[5] = {FS_FIELD_PHI, FS_FIELD_U, FS_FIELD_V, FS_FIELD_W, FS_FIELD_PRESSURE};
  for (int fld : fields) {
    if (!ok) break;
    std::vector<double> a((size_t)field_count(c, fld));
    fs_status st = fs_download(c, fld, a.data(), nullptr);
    if (st != FS_OK) { std::fclose(f); return st; }
    ok = std::fwrite(a.data(), sizeof(double), a.size(), f) == a.size();
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) { set_error("short write to %s", path); return FS_INVALID_ARG; }
  return FS_OK;
}

fs_status fs_read_state(fs_ctx* c, const char* path) {
  if (!c || !path) { set_error("NULL argument"); return FS_INVALID_ARG; }
  FILE* f = std::fopen(path, "rb");
  if (!f) { set_error("cannot open %s", path); return FS_INVALID_ARG; }
  char magic[8];
  uint32_t version = 0;
  int32_t dims[3];
  double dx = 0.0;
  bool ok = std::fread(magic, 8, 1, f) == 1 && std::memcmp(magic, kStateMagic, 8) == 0 &&
            std::fread(&version, 4, 1, f) == 1 && version == 1 && std::fread(dims, sizeof dims, 1, f) == 1 &&
            std::fread(&dx, 8, 1, f) == 1;
  if (!ok) { std::fclose(f); set_error("%s is not a state file of this library", path); return FS_INVALID_ARG; }
  if (dims[0] != c->grid.nx || dims[1] != c->grid.ny || dims[2] != c->grid.nz || dx != c->grid.dx) {
    std::fclose(f);
    set_error("%s holds a %d x %d x %d grid with dx %.17g, not the context's", path, dims[0], dims[1], dims[2], dx);
    return FS_INVALID_ARG;
  }
  const int fields[5] = {FS_FIELD_PHI, FS_FIELD_U, FS_FIELD_V, FS_FIELD_W, FS_FIELD_PRESSURE};
  std::vector<std::vector<double>> data(5);
  for (int q = 0; q < 5 && ok; ++q) {
    data[q].resize((size_t)field_count(c, fields[q]));
    ok = std::fread(data[q].data(), sizeof(double), data[q].size(), f) == data[q].size();
  }
  std::fclose(f);
  if (!ok) { set_error("%s is truncated", path); return FS_INVALID_ARG; }
  for (int q = 0; q < 5; ++q) CKS(fs_upload(c, fields[q], data[q].data(), nullptr));
  return FS_OK;
}

// ---- adjoints (corrected projection; FP64 bars over FP64 or FP32 states)

fs_status fs_adjoint_reset(fs_ctx* c) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  CKS(adj_check(c));
  CKS(zero_cell(c, c->abar[0]));
  CKS(zero_faces(c, &c->abar[1]));
  CK(cudaMemsetAsync(c->a_rho, 0, 4 * sizeof(double), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_adjoint_density_bars(fs_ctx* c, double* rho_neg_bar, double* rho_pos_bar) {
  if (!c || !rho_neg_bar || !rho_pos_bar) { set_error("NULL argument"); return FS_INVALID_ARG; }
  CKS(adj_check(c));
  CK(cudaMemcpyAsync(c->sc_host, c->a_rho, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *rho_neg_bar = c->sc_host[0];
  *rho_pos_bar = c->sc_host[1];
  return FS_OK;
}

// The status of an adjoint entry point: a transposed solve that stopped
// before its tolerance (iteration cap, stagnation) makes the bars inexact;
// the call completes and reports FS_NOT_CONVERGED.
static fs_status adj_finish(fs_ctx* c, fs_status s) {
  if (s == FS_OK && c->adj_unconverged > 0) {
    char msg[320];
    std::snprintf(msg, sizeof msg, "%d adjoint solve(s) stopped before their tolerance (last: %s)", c->adj_unconverged,
                  c->adj_note);
    set_error(msg);
    return FS_NOT_CONVERGED;
  }
  return s;
}

static void adj_begin(fs_ctx* c) {
  c->adj_unconverged = 0;
  c->adj_worst_rel = 0.0;
  c->adj_note[0] = 0;
}

fs_status fs_step_adjoint(fs_ctx* c, double dt, fs_step_report* rep) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  CKS(box_only(c, "fs_step_adjoint"));
  if (!(dt > 0) || !std::isfinite(dt)) { set_error("dt must be positive and finite"); return FS_INVALID_ARG; }
  CKS(adj_check(c));
  fs_step_report local{};
  fs_step_report* r = rep ? rep : &local;
  *r = fs_step_report{};
  c->launches = 0;
  c->pcg_ms = 0.0f;
  c->pcg_launched_iterations = 0;
  CKS(timed_begin(c));
  adj_begin(c);
  fs_status s = c->fp32 ? step_adjoint_t<float>(c, dt, r) : step_adjoint_t<double>(c, dt, r);
  if (s != FS_OK && s != FS_NOT_CONVERGED) return s;
  CKS(timed_end(c, &r->ms));
  r->pcg_ms = c->pcg_ms;
  r->pcg_launched_iterations = c->pcg_launched_iterations;
  r->kernel_launches = c->launches;
  return adj_finish(c, s);
}

fs_status fs_advect_levelset_adjoint(fs_ctx* c, double dt) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  CKS(box_only(c, "fs_advect_levelset_adjoint"));
  CKS(adj_check(c));
  void* vel[3] = {c->u, c->v, c->w};
  CKS(c->fp32 ? adj_levelset_fe<float>(c, c->phi, vel, c->abar[0], 1.0, c->awork_c[0], &c->abar[1], dt)
              : adj_levelset_fe<double>(c, c->phi, vel, c->abar[0], 1.0, c->awork_c[0], &c->abar[1], dt));
  CKS(copy_cell(c, c->abar[0], c->awork_c[0]));
  CK(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_advect_velocity_adjoint(fs_ctx* c, double dt) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  CKS(box_only(c, "fs_advect_velocity_adjoint"));
  CKS(adj_check(c));
  void* vel[3] = {c->u, c->v, c->w};
  CKS(c->fp32 ? adj_velocity_advect<float>(c, vel, &c->abar[1], c->awork_f[0], dt)
              : adj_velocity_advect<double>(c, vel, &c->abar[1], c->awork_f[0], dt));
  CKS(copy_faces(c, &c->abar[1], c->awork_f[0]));
  CK(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_reinitialize_adjoint(fs_ctx* c) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  CKS(box_only(c, "fs_reinitialize_adjoint"));
  CKS(adj_check(c));
  Tape tp;
  CKS(tape_bind(c, &tp));
  if (c->fp32) {
    CKS(reinit_block_t<float>(c, c->phi, c->s1, c->phi, 0.0, 1.0, c->s2, c->s3, &tp.re[0]));
    CKS(adj_reinit_block<float>(c, tp.re[0], c->abar[0], c->awork_c[0]));
  } else {
    CKS(reinit_block_t<double>(c, c->phi, c->s1, c->phi, 0.0, 1.0, c->s2, c->s3, &tp.re[0]));
    CKS(adj_reinit_block<double>(c, tp.re[0], c->abar[0], c->awork_c[0]));
  }
  CKS(copy_cell(c, c->abar[0], c->awork_c[0]));
  CK(cudaStreamSynchronize(c->stream));
  return FS_OK;
}

fs_status fs_viscosity_adjoint(fs_ctx* c, double dt) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  CKS(box_only(c, "fs_viscosity_adjoint"));
  if (!(dt > 0)) { set_error("dt must be positive"); return FS_INVALID_ARG; }
  CKS(adj_check(c));
  if (c->prm.viscosity != 1) { set_error("the semi-implicit viscosity is off"); return FS_INVALID_ARG; }
  Tape tp;
  CKS(tape_bind(c, &tp));
  adj_begin(c);
  CKS(tape_velocity(c, tp.vel[0][1]));
  CKS(c->fp32 ? viscosity_t<float>(c, dt, nullptr) : viscosity_t<double>(c, dt, nullptr));
  CKS(tape_velocity(c, tp.vel[0][2]));
  void* vel[3] = {c->u, c->v, c->w};
  CKS(copy_fields(c, vel, tp.vel[0][1]));  // the context keeps the operator's input
  CKS(c->fp32 ? adj_viscosity<float>(c, c->phi, tp.vel[0][1], tp.vel[0][2], &c->abar[1], c->awork_f[1], c->abar[0], dt)
              : adj_viscosity<double>(c, c->phi, tp.vel[0][1], tp.vel[0][2], &c->abar[1], c->awork_f[1], c->abar[0],
                                      dt));
  CKS(copy_faces(c, &c->abar[1], c->awork_f[1]));
  CK(cudaStreamSynchronize(c->stream));
  return adj_finish(c, FS_OK);
}

fs_status fs_project_adjoint(fs_ctx* c, double dt) {
  if (!c) { set_error("NULL context"); return FS_INVALID_ARG; }
  CKS(box_only(c, "fs_project_adjoint"));
  if (!(dt > 0) || !std::isfinite(dt)) { set_error("dt must be positive and finite"); return FS_INVALID_ARG; }
  CKS(adj_check(c));
  Tape tp;
  CKS(tape_bind(c, &tp));
  adj_begin(c);
  CKS(tape_velocity(c, tp.vel[0][2]));
  fs_status s = c->fp32 ? project_t<float>(c, dt, 0.0, 1.0, nullptr) : project_t<double>(c, dt, 0.0, 1.0, nullptr);
  if (s != FS_OK && s != FS_NOT_CONVERGED) return s;
  CKS(copy_cell(c, tp.p[0], c->p64));
  void* vel[3] = {c->u, c->v, c->w};
  CKS(copy_fields(c, vel, tp.vel[0][2]));  // the context keeps the operator's input
  CKS(c->fp32 ? adj_projection<float>(c, c->phi, tp.vel[0][2], tp.p[0], &c->abar[1], 1.0, c->awork_f[1], c->abar[0], dt)
              : adj_projection<double>(c, c->phi, tp.vel[0][2], tp.p[0], &c->abar[1], 1.0, c->awork_f[1], c->abar[0],
                                       dt));
  CKS(copy_faces(c, &c->abar[1], c->awork_f[1]));
  CK(cudaStreamSynchronize(c->stream));
  return adj_finish(c, s);
}

fs_status fs_pcg_csr(fs_ctx* c, int n, int nnz, const double* values, const int* column_index, const int* row_ptr,
                     const double* b, double* x, double tolerance, int max_iteration, int stop, int* iterations,
                     double* residual);

}  // extern "C"
