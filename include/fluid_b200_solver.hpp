// fluid_b200_solver.hpp - C++ host mirror of the reference solver's
// interface for the timestep path, over the C ABI of fluid_b200.h.
//
// Class names, method names, argument meaning and script keys follow the
// reference (EULERIAN_FLUID_SOLVER_3D.h, PROJECTION_3D.h, LINEAR_SOLVER.h,
// SCRIPT_READER.h), so code written against the reference reads the same;
// the bodies call the device-resident library.  The reference runs every
// method on all worker threads with a barrier after each loop
// (MULTITHREADING.h); here the work happens once, on thread_id 0 (the
// reference's BEGIN_HEAD_THREAD_WORK), and calls from other thread ids return
// at once.  Failures throw fluid_b200::Error carrying the fs_status and the
// library's message, where the reference would assert or exit().
//
// Header only; link with libfluidb200.so.  C++17.
#ifndef FLUID_B200_SOLVER_HPP
#define FLUID_B200_SOLVER_HPP

#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "fluid_b200.h"

namespace fluid_b200 {

class Error : public std::runtime_error {
 public:
  Error(fs_status s, const std::string& where)
      : std::runtime_error(where + ": " + fs_status_str(s) + ": " + fs_last_error()), status(s) {}
  fs_status status;
};

inline fs_status check(fs_status s, const char* where, bool allow_not_converged = false) {
  if (s == FS_OK || (allow_not_converged && s == FS_NOT_CONVERGED)) return s;
  throw Error(s, where);
}

// ---------------------------------------------------------------------------
// .sim scripts (SCRIPT_READER.h:161-173): named blocks in braces, key = value
// assignments (numbers without exponent, true/false, quoted strings,
// parenthesised vectors), // and /* */ comments; "// NAME {" comments out the
// whole block.  Getters return the default when the key is absent.
// ---------------------------------------------------------------------------
class SCRIPT_BLOCK {
 public:
  std::string name;
  std::map<std::string, std::string> values;
  std::vector<SCRIPT_BLOCK> blocks;

  const SCRIPT_BLOCK& FindBlock(const std::string& n) const {
    for (const auto& b : blocks)
      if (b.name == n) return b;
    static const SCRIPT_BLOCK empty;
    return empty;
  }
  double GetFloat(const std::string& key, double def = 0.0) const {
    auto it = values.find(key);
    return it == values.end() ? def : number(it->second, key);
  }
  int GetInteger(const std::string& key, int def = 0) const { return (int)GetFloat(key, def); }
  bool GetBoolean(const std::string& key, bool def = false) const {
    auto it = values.find(key);
    if (it == values.end()) return def;
    if (it->second != "true" && it->second != "false") throw std::invalid_argument(key + ": expected true/false");
    return it->second == "true";
  }
  std::string GetString(const std::string& key, const std::string& def = "") const {
    auto it = values.find(key);
    if (it == values.end()) return def;
    const std::string& v = it->second;
    return (v.size() >= 2 && v.front() == '"') ? v.substr(1, v.size() - 2) : v;
  }
  void GetVector3(const std::string& key, double out[3], const double def[3]) const {
    auto it = values.find(key);
    if (it == values.end()) {
      for (int a = 0; a < 3; ++a) out[a] = def[a];
      return;
    }
    std::string v = it->second;
    if (v.size() < 2 || v.front() != '(' || v.back() != ')') throw std::invalid_argument(key + ": expected (a, b, c)");
    v = v.substr(1, v.size() - 2);
    std::vector<std::string> parts;
    std::stringstream ss(v);
    std::string p;
    while (std::getline(ss, p, ',')) parts.push_back(p);
    if (parts.size() != 3) throw std::invalid_argument(key + ": expected a 3-vector");
    for (int a = 0; a < 3; ++a) out[a] = number(parts[a], key);
  }

  // the script syntax: minus signs, digits, at most one '.', no exponent
  static double number(const std::string& text, const std::string& key) {
    std::string t;
    for (char ch : text)
      if (!std::isspace((unsigned char)ch)) t += ch;
    size_t q = 0;
    int minus = 0;
    while (q < t.size() && t[q] == '-') ++minus, ++q;
    const std::string body = t.substr(q);
    int dots = 0, digits = 0;
    for (char ch : body) {
      if (ch == '.') ++dots;
      else if (std::isdigit((unsigned char)ch)) ++digits;
      else digits = -1000;
    }
    if (body.empty() || dots > 1 || digits <= 0 || body.back() == '.')
      throw std::invalid_argument(key + ": '" + text + "' is not a number in the script syntax");
    const double v = std::strtod(body.c_str(), nullptr);
    return (minus % 2) ? -v : v;
  }
};

class SCRIPT_READER {
 public:
  explicit SCRIPT_READER(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open script " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    Parse(ss.str());
  }
  static SCRIPT_READER FromText(const std::string& text) {
    SCRIPT_READER r;
    r.Parse(text);
    return r;
  }
  const SCRIPT_BLOCK& FindBlock(const std::string& name) const { return root.FindBlock(name); }
  SCRIPT_BLOCK root;

 private:
  SCRIPT_READER() = default;
  enum Kind { WORD, LINE_COMMENT };
  std::vector<std::pair<Kind, std::string>> tokens_;

  void Tokenize(const std::string& s) {
    size_t i = 0;
    while (i < s.size()) {
      const char ch = s[i];
      if (std::isspace((unsigned char)ch)) { ++i; continue; }
      if (s.compare(i, 2, "//") == 0) {
        tokens_.push_back({LINE_COMMENT, ""});
        while (i < s.size() && s[i] != '\n') ++i;
        continue;
      }
      if (s.compare(i, 2, "/*") == 0) {
        const size_t e = s.find("*/", i + 2);
        i = e == std::string::npos ? s.size() : e + 2;
        continue;
      }
      if (ch == '"') {
        const size_t e = s.find('"', i + 1);
        if (e == std::string::npos) throw std::invalid_argument("unterminated string in script");
        tokens_.push_back({WORD, s.substr(i, e - i + 1)});
        i = e + 1;
        continue;
      }
      if (ch == '(') {
        const size_t e = s.find(')', i + 1);
        if (e == std::string::npos) throw std::invalid_argument("unterminated vector in script");
        tokens_.push_back({WORD, s.substr(i, e - i + 1)});
        i = e + 1;
        continue;
      }
      if (ch == '{' || ch == '}' || ch == '=') {
        tokens_.push_back({WORD, std::string(1, ch)});
        ++i;
        continue;
      }
      size_t e = i;
      while (e < s.size() && !std::isspace((unsigned char)s[e]) && s[e] != '{' && s[e] != '}' && s[e] != '=' &&
             s[e] != '(' && s[e] != ')' && s[e] != '"')
        ++e;
      if (e == i) throw std::invalid_argument("unbalanced ')' in script");
      tokens_.push_back({WORD, s.substr(i, e - i)});
      i = e;
    }
  }

  size_t SkipBlock(size_t pos) const {
    int depth = 0;
    for (; pos < tokens_.size(); ++pos) {
      if (tokens_[pos].first != WORD) continue;
      if (tokens_[pos].second == "{") ++depth;
      if (tokens_[pos].second == "}" && --depth == 0) return pos + 1;
    }
    throw std::invalid_argument("commented-out block is not closed");
  }

  size_t ParseBlock(size_t pos, SCRIPT_BLOCK& b) {
    while (pos < tokens_.size()) {
      if (tokens_[pos].first == LINE_COMMENT) {
        ++pos;
        if (pos < tokens_.size() && tokens_[pos].first == WORD && tokens_[pos].second == "{") pos = SkipBlock(pos);
        continue;
      }
      const std::string& tok = tokens_[pos].second;
      if (tok == "}") return pos + 1;
      if (pos + 1 < tokens_.size() && tokens_[pos + 1].second == "{") {
        SCRIPT_BLOCK child;
        child.name = tok;
        pos = ParseBlock(pos + 2, child);
        b.blocks.push_back(std::move(child));
        continue;
      }
      if (pos + 2 < tokens_.size() && tokens_[pos + 1].second == "=") {
        b.values[tok] = tokens_[pos + 2].second;
        pos += 3;
        continue;
      }
      throw std::invalid_argument("unexpected token '" + tok + "' in block '" + b.name + "'");
    }
    if (!b.name.empty()) throw std::invalid_argument("block '" + b.name + "' is not closed");
    return pos;
  }

  void Parse(const std::string& text) {
    Tokenize(text);
    ParseBlock(0, root);
  }
};

// ---------------------------------------------------------------------------
// grid, matrix, linear solver plugin
// ---------------------------------------------------------------------------
struct GRID_STRUCTURE_3D {  // GRID_STRUCTURE_3D.h:91-137: dx = (max - min)/(res - 1)
  int i_res = 1, j_res = 1, k_res = 1;
  double x_min = 0, y_min = 0, z_min = 0, x_max = 1, y_max = 1, z_max = 1;
  double dx = 1, dy = 1, dz = 1;

  void Initialize(int ir, int jr, int kr, const double mn[3], const double mx[3]) {
    i_res = ir; j_res = jr; k_res = kr;
    x_min = mn[0]; y_min = mn[1]; z_min = mn[2];
    x_max = mx[0]; y_max = mx[1]; z_max = mx[2];
    dx = (x_max - x_min) / (i_res > 1 ? i_res - 1 : 1);
    dy = (y_max - y_min) / (j_res > 1 ? j_res - 1 : 1);
    dz = (z_max - z_min) / (k_res > 1 ? k_res - 1 : 1);
  }
  void InitializeFromBlock(const SCRIPT_BLOCK& b) {
    const double one[3] = {1, 1, 1}, zero[3] = {0, 0, 0};
    double res[3], mn[3], mx[3];
    b.GetVector3("base_grid_resolution", res, one);
    b.GetVector3("base_grid_min", mn, zero);
    b.GetVector3("base_grid_max", mx, one);
    if (b.GetFloat("resolution_scale", 1.0) != 1.0) throw std::invalid_argument("resolution_scale != 1 is not supported");
    Initialize((int)res[0], (int)res[1], (int)res[2], mn, mx);
  }
};

template <class TT> struct CSR_MATRIX {  // CSR_MATRIX.h:10-35
  int N = 0, nz = 0;
  std::vector<TT> values;
  std::vector<int> column_index, row_ptr;
};

template <class TT> struct VECTOR_ND {  // VECTOR_ND.h:7-12: num_dimension values
  int num_dimension = 0;
  std::vector<TT> values;
  VECTOR_ND() = default;
  explicit VECTOR_ND(int n, TT v = TT(0)) : num_dimension(n), values(n, v) {}
  TT& operator[](int i) { return values[i]; }
  const TT& operator[](int i) const { return values[i]; }
};

// The boundary-condition tags the reference passes to every linear solver
// (FIELD_STRUCTURE_3D<int> bc, one tag per cell); the Jacobi-PCG does not
// read them (PCG_METHOD.h: Solve hands A, x, b to PCGMethod).
template <class TT> struct FIELD_STRUCTURE_3D {
  GRID_STRUCTURE_3D grid;
  std::vector<TT> values;
};

class LINEAR_SOLVER {  // LINEAR_SOLVER.h:36: Solve is the plugin point
 public:
  virtual ~LINEAR_SOLVER() = default;
  double tolerance = 1.0, sqr_tolerance = 1.0, residual = 1e8;
  int max_iteration = 10, num_iteration = 0;

  void Initialize(double tol, int max_it) {
    max_iteration = max_it;
    SetTolerance(tol);
  }
  void SetTolerance(double tol) {
    tolerance = tol;
    sqr_tolerance = tol * tol;
  }
  virtual void Solve(const int& thread_id, const CSR_MATRIX<double>& A, VECTOR_ND<double>& x,
                     const VECTOR_ND<double>& b, const FIELD_STRUCTURE_3D<int>& bc) = 0;
};

// Jacobi-PCG on the GPU with the reference's stopping test r.z < tol^2
// (PCG_METHOD.cpp:87), or ||r||/||b|| < tol with relative = true.
class CUDA_PCG_METHOD : public LINEAR_SOLVER {
 public:
  explicit CUDA_PCG_METHOD(bool rel = false) : relative(rel) {}
  bool relative;
  void Solve(const int& thread_id, const CSR_MATRIX<double>& A, VECTOR_ND<double>& x, const VECTOR_ND<double>& b,
             const FIELD_STRUCTURE_3D<int>& bc) override {
    (void)bc;  // boundary tags: already folded into A by the system builder
    if (thread_id != 0) return;
    if (x.num_dimension != A.N || b.num_dimension != A.N || (int)x.values.size() != A.N ||
        (int)b.values.size() != A.N)
      throw std::invalid_argument("CUDA_PCG_METHOD: size mismatch");
    int it = 0;
    double res = 0.0;
    check(fs_pcg_csr(nullptr, A.N, A.nz, A.values.data(), A.column_index.data(), A.row_ptr.data(), b.values.data(),
                     x.values.data(), tolerance, max_iteration, relative ? FS_STOP_RELATIVE : FS_STOP_ABSOLUTE, &it,
                     &res),
          "fs_pcg_csr", true);
    num_iteration = it;
    residual = res;
  }
};

// fs_params from a FLUID_SOLVER_UNIFORM_AIR_WATER block, keys and defaults
// as EULERIAN_FLUID_SOLVER_3D.h:192-260 and PROJECTION_3D.h:178-230 read
// them; new keys: precision ("fp64" or "fp32_refine"), relative_tolerance,
// semi_implicit_approach, viscosity_tolerance, corrected_projection.
inline fs_params params_from_block(const SCRIPT_BLOCK& block, const GRID_STRUCTURE_3D& grid) {
  const SCRIPT_BLOCK& proj = block.FindBlock("PROJECTION_WATER");
  const SCRIPT_BLOCK& adv = block.FindBlock("LEVELSET_ADVECTION");
  const bool water_drop = proj.GetBoolean("water_drop", false), bubble = proj.GetBoolean("air_bubble_rising", false);
  if (water_drop == bubble)
    throw std::invalid_argument("exactly one of PROJECTION_WATER.water_drop / air_bubble_rising must be true");
  const double wd = block.GetFloat("water_density", 1.0), ad = block.GetFloat("air_density", 1.0);
  const double wv = block.GetFloat("water_viscosity", 1.0), av = block.GetFloat("air_viscosity", 0.0);
  fs_params p;
  fs_params_default(&p);
  p.rho_neg = water_drop ? wd : ad;
  p.mu_neg = water_drop ? wv : av;
  p.rho_pos = water_drop ? ad : wd;
  p.mu_pos = water_drop ? av : wv;
  const double g_def[3] = {0.0, -9.8, 0.0};
  block.GetVector3("gravity", p.gravity, g_def);
  p.weno_epsilon = adv.GetFloat("epsilon", 10e-6);
  // EULERIAN_FLUID_SOLVER_3D.h:201-202, 2198-2225: Sussman pseudo-steps only with
  // sussmanstyle_reinitialization, fast sweeping before them with
  // fastsweeping_reinitialization (both default false)
  p.reinit_iterations = block.GetBoolean("sussmanstyle_reinitialization", false)
                            ? block.GetInteger("iteration_number_for_reinitialization", 10)
                            : 0;
  p.fast_sweeping = block.GetBoolean("fastsweeping_reinitialization", false) ? 1 : 0;
  p.reinit_scaling = block.GetInteger("scaling_number_for_reinitialization", 5);
  p.order = block.GetInteger("order_for_time_advancing", 1);
  const std::string prec = block.GetString("precision", "fp64");
  if (prec != "fp64" && prec != "fp32_refine") throw std::invalid_argument("precision must be fp64 or fp32_refine");
  p.precision = prec == "fp32_refine" ? FS_PRECISION_FP32_REFINE : FS_PRECISION_FP64;
  p.stop = proj.GetBoolean("relative_tolerance", false) ? FS_STOP_RELATIVE : FS_STOP_ABSOLUTE;
  p.tolerance = proj.GetFloat("tolerance", 1e-4);
  p.max_iteration = proj.GetInteger("max_iteration", 30);
  p.inner_tolerance = proj.GetFloat("inner_tolerance", 1e-2);
  p.max_outer = proj.GetInteger("max_outer", 20);
  // semi_implicit_approach = false: the reference's air/water explicit update
  p.viscosity = block.GetBoolean("semi_implicit_approach", true) ? 1 : 2;
  p.viscosity_tolerance = block.GetFloat("viscosity_tolerance", 1e-8);
  p.flags = block.GetBoolean("corrected_projection", true) ? 0 : FS_FLAG_FAITHFUL_PROJECTION;
  p.surface_tension = block.GetFloat("surface_tension", 0.0);
  // VELOCITY_ADVECTION (ADVECTION_3D.h:109-112, 317-328): ENO3 when only
  // use_3rd_eno_v is set, else WENO5; with both set the reference applies both
  // in one stage, which is refused.
  const SCRIPT_BLOCK& vel = block.FindBlock("VELOCITY_ADVECTION");
  const bool weno_v = vel.GetBoolean("use_5th_weno_v", false), eno_v = vel.GetBoolean("use_3rd_eno_v", false);
  if (weno_v && eno_v) throw std::invalid_argument("VELOCITY_ADVECTION selects both use_5th_weno_v and use_3rd_eno_v");
  p.velocity_scheme = eno_v ? FS_VELOCITY_ENO3 : FS_VELOCITY_WENO5;
  p.velocity_epsilon = vel.GetFloat("epsilon", 10e-6);
  if (p.precision == FS_PRECISION_FP32_REFINE) p.stop = FS_STOP_RELATIVE;
  if (std::abs(grid.dx - grid.dy) > 1e-12 * grid.dx || std::abs(grid.dx - grid.dz) > 1e-12 * grid.dx)
    throw std::invalid_argument("the solver needs a uniform grid (dx = dy = dz)");
  return p;
}

// fs_params for the reference's oil/water vertical pipe from its
// SIMULATION_WORLD block (a, R2, CFL; SIMULATION_WORLD.h:119-125) and
// FLUID_SOLVER_UNIFORM_OIL_WATER block, with the dimensionless constants the
// reference derives (EULERIAN_FLUID_SOLVER_3D.h:496-514): R1 = R2/a,
// f = g (oil - K water)/(K - 1), A = (a^2 - 1) + (m K + 2 (K - 1) ln a),
// V0 = (f + water g) R1^2/(4 water_viscosity) A, J = sigma R1 oil/
// oil_viscosity^2, Re = oil R1 |V0|/oil_viscosity, We = Re^2/J.  The
// operators run as the reference's do; the pipe's viscosity is not built, so
// the script must switch the sourcing step off (is_sourcing_active = false).
inline fs_params pipe_params_from_script(const SCRIPT_BLOCK& world, const SCRIPT_BLOCK& block,
                                         const GRID_STRUCTURE_3D& grid) {
  if (block.GetBoolean("is_sourcing_active", true))
    throw std::invalid_argument("the pipe mode's viscosity is not built: set is_sourcing_active = false");
  if (!block.GetBoolean("dimensionless_form", false))
    throw std::invalid_argument("the pipe mode is built for dimensionless_form = true");
  if (block.FindBlock("VELOCITY_ADVECTION").GetBoolean("use_5th_weno_v", false))
    throw std::invalid_argument("the pipe mode advects the velocity with ENO3 (use_3rd_eno_v) only");
  const double a = world.GetFloat("a", 1.0), R2 = world.GetFloat("R2", 1.0);
  const double m = block.GetFloat("m", 1.0), eta = block.GetFloat("eta", 1.0);
  const double K = block.GetFloat("K", 1.0), g = block.GetFloat("g", 1.0);
  const double wd = block.GetFloat("water_density", 1.0), od = block.GetFloat("oil_density", 1.0);
  const double wv = block.GetFloat("water_viscosity", 1.0), ov = block.GetFloat("oil_viscosity", 0.0);
  const double sigma = block.GetFloat("surface_tension", 0.0);
  const double R1 = R2 / a;
  const double f = 1.0 / (K - 1.0) * g * (od - K * wd);
  const double A = (a * a - 1.0) + (m * K + 2.0 * (K - 1) * std::log(a));
  const double V0 = (f + wd * g) * (R1 * R1) / (4.0 * wv) * A;
  const double J = sigma * R1 * od / (ov * ov);
  const double Re = (od * R1 * std::abs(V0)) / ov;
  const double We = (1.0 / J) * (Re * Re);
  const SCRIPT_BLOCK& proj = block.FindBlock("PROJECTION_WATER");
  fs_params p;
  fs_params_default(&p);
  p.pipe = 1;
  p.pipe_radius = a;
  p.grid_min[0] = grid.x_min; p.grid_min[1] = grid.y_min; p.grid_min[2] = grid.z_min;
  p.grid_max[0] = grid.x_max; p.grid_max[1] = grid.y_max; p.grid_max[2] = grid.z_max;
  p.pipe_R1 = R1;
  p.pipe_V0 = V0;
  p.pipe_f = f;
  p.pipe_eta = eta;
  p.pipe_oil_density = od;
  p.pipe_We = We;
  p.rho_neg = 1.0;
  p.rho_pos = wd / od;
  const double g_def[3] = {0.0, -9.8, 0.0};
  block.GetVector3("gravity", p.gravity, g_def);
  p.weno_epsilon = block.FindBlock("LEVELSET_ADVECTION").GetFloat("epsilon", 10e-6);
  p.reinit_iterations = block.GetBoolean("sussmanstyle_reinitialization", false)
                            ? block.GetInteger("iteration_number_for_reinitialization", 10)
                            : 0;
  p.reinit_scaling = block.GetInteger("scaling_number_for_reinitialization", 5);
  p.order = block.GetInteger("order_for_time_advancing", 1);
  p.stop = FS_STOP_ABSOLUTE;
  p.tolerance = proj.GetFloat("tolerance", 1e-4);
  p.max_iteration = proj.GetInteger("max_iteration", 30);
  p.viscosity = 0;
  p.flags = FS_FLAG_FAITHFUL_PROJECTION | FS_FLAG_REINIT_TYPO | FS_FLAG_CURVATURE_TYPO;
  p.velocity_scheme = FS_VELOCITY_ENO3;
  p.cfl = world.GetFloat("CFL", 0.5);
  return p;
}

// ---------------------------------------------------------------------------
// solver classes
// ---------------------------------------------------------------------------
class PROJECTION_3D {  // PROJECTION_3D.h:416
 public:
  explicit PROJECTION_3D(fs_ctx* c) : ctx_(c) {}
  fs_solve_report last_report{};
  fs_status last_status = FS_OK;

  void Solve(const int& thread_id, const double& dt) {
    if (thread_id != 0) return;
    last_status = check(fs_project(ctx_, dt, &last_report), "fs_project", true);
  }
  std::vector<double> pressure_field() const { return download(FS_FIELD_PRESSURE); }
  std::vector<double> divergence_field() const { return download(FS_FIELD_DIVERGENCE); }

 private:
  fs_ctx* ctx_;
  std::vector<double> download(int field) const;
  friend class EULERIAN_FLUID_SOLVER_3D;
  int nx_ = 0, ny_ = 0, nz_ = 0;
};

class EULERIAN_FLUID_SOLVER_3D {  // EULERIAN_FLUID_SOLVER_3D.h
 public:
  EULERIAN_FLUID_SOLVER_3D() = default;
  EULERIAN_FLUID_SOLVER_3D(const EULERIAN_FLUID_SOLVER_3D&) = delete;
  EULERIAN_FLUID_SOLVER_3D& operator=(const EULERIAN_FLUID_SOLVER_3D&) = delete;
  ~EULERIAN_FLUID_SOLVER_3D() {
    if (ctx_) fs_destroy(ctx_);
  }

  GRID_STRUCTURE_3D base_grid;
  std::unique_ptr<PROJECTION_3D> water_projection;
  int order_for_time_advancing = 1;
  fs_step_report last_report{};
  fs_status last_status = FS_OK;

  // EULERIAN_FLUID_SOLVER_3D.h:192 (the MULTITHREADING argument is not needed)
  void InitializeFromScriptBlock(const GRID_STRUCTURE_3D& world_grid, const SCRIPT_BLOCK& fluid_solver_block) {
    base_grid = world_grid;
    fs_params p = params_from_block(fluid_solver_block, world_grid);
    order_for_time_advancing = p.order;
    Create(p);
  }
  void Create(const fs_params& p) {
    if (ctx_) fs_destroy(ctx_);
    ctx_ = nullptr;
    fs_grid_desc g{base_grid.i_res, base_grid.j_res, base_grid.k_res, base_grid.dx};
    check(fs_create(&g, &p, &ctx_), "fs_create");
    water_projection.reset(new PROJECTION_3D(ctx_));
    water_projection->nx_ = g.nx;
    water_projection->ny_ = g.ny;
    water_projection->nz_ = g.nz;
    params_ = p;
  }
  // a .sim script (SIMULATION_WORLD.h:InitializeFromScript): the air/water
  // box, or the oil/water vertical pipe with its sourcing step off
  // (pipe_params_from_script); pipe scripts that need the pipe's viscosity,
  // and horizontal pipes, are refused rather than run wrong
  void InitializeFromScript(const std::string& path) {
    SCRIPT_READER r(path);
    const SCRIPT_BLOCK& world = r.FindBlock("SIMULATION_WORLD");
    if (world.GetBoolean("oil_water_simulation", false)) {
      const SCRIPT_BLOCK& disc = world.FindBlock("WORLD_DISCRETIZATION_OIL_WATER");
      if (!disc.FindBlock("PIPE_OPTIONS").GetBoolean("is_vertical", false))
        throw std::invalid_argument("the pipe mode is built for the vertical pipe (PIPE_OPTIONS.is_vertical) only");
      GRID_STRUCTURE_3D g;
      g.InitializeFromBlock(disc.FindBlock("GRID_STRUCTURE_3D_VERTICAL"));
      base_grid = g;
      const fs_params p = pipe_params_from_script(world, r.FindBlock("FLUID_SOLVER_UNIFORM_OIL_WATER"), g);
      order_for_time_advancing = p.order;
      Create(p);
      return;
    }
    GRID_STRUCTURE_3D g;
    g.InitializeFromBlock(world.FindBlock("WORLD_DISCRETIZATION_AIR_WATER").FindBlock("GRID_STRUCTURE_3D_LARGE"));
    InitializeFromScriptBlock(g, r.FindBlock("FLUID_SOLVER_UNIFORM_AIR_WATER"));
    params_.cfl = world.GetFloat("CFL", 0.5);
    check(fs_set_params(ctx_, &params_), "fs_set_params");
  }

  // fields: interior values, x fastest (ARRAY_3D.h:98); faces carry one more
  // entry along their own axis
  void SetField(int field, const std::vector<double>& a) {
    if ((int64_t)a.size() != Count(field)) throw std::invalid_argument("SetField: wrong size");
    check(fs_upload(ctx_, field, a.data(), nullptr), "fs_upload");
  }
  std::vector<double> GetField(int field) const {
    std::vector<double> a((size_t)Count(field));
    check(fs_download(ctx_, field, a.data(), nullptr), "fs_download");
    return a;
  }
  int64_t Count(int field) const {
    const int64_t n = (int64_t)base_grid.i_res * base_grid.j_res * base_grid.k_res;
    switch (field) {
      case FS_FIELD_U: return n / base_grid.i_res * (base_grid.i_res + 1);
      case FS_FIELD_V: return n / base_grid.j_res * (base_grid.j_res + 1);
      case FS_FIELD_W: return n / base_grid.k_res * (base_grid.k_res + 1);
      default: return n;
    }
  }

  // EULERIAN_FLUID_SOLVER_3D.h:803
  void AdvanceOneTimeStepThread(const int& thread_id, const double& dt) {
    if (thread_id != 0) return;
    last_status = check(fs_step(ctx_, dt, &last_report), "fs_step", true);
  }
  // dt limit before the CFL factor (the reference multiplies by CFL in SIMULATION_WORLD)
  double CFLOneTimeStep() const {
    double dt = 0.0;
    check(fs_cfl_dt(ctx_, &dt), "fs_cfl_dt");
    return dt / params_.cfl;
  }
  double CFL() const { return params_.cfl; }
  fs_ctx* context() const { return ctx_; }

  // water_levelset->ReinitializeByFastSweeping (LEVELSET_3D.h:601): the
  // context's sweep direction, which then advances
  void ReinitializeByFastSweeping(const int& thread_id) {
    if (thread_id != 0) return;
    check(fs_fast_sweeping(ctx_, -1, 1), "fs_fast_sweeping");
  }
  // water_levelset->FullFastSweepingMethodThreaded (LEVELSET_3D.h:828-835):
  // four calls in sweep directions 0..3, each starting from its own set-up
  // (corrected = true: one set-up, then all eight sweeps)
  void FullFastSweepingMethodThreaded(bool corrected = false) {
    if (corrected) {
      check(fs_fast_sweeping(ctx_, 0, 4), "fs_fast_sweeping");
      return;
    }
    for (int d = 0; d < 4; ++d) check(fs_fast_sweeping(ctx_, d, 1), "fs_fast_sweeping");
  }

 private:
  fs_ctx* ctx_ = nullptr;
  fs_params params_{};
};

// WRITE_LEVELSET (WRITE_LEVELSET.h:8-84): the water level set's surface as
// an OBJ file; the caller names the file (the reference derives it from the
// frame number and its output directory).
class WRITE_LEVELSET {
 public:
  explicit WRITE_LEVELSET(const EULERIAN_FLUID_SOLVER_3D& solver) : solver_(solver) {}
  void WriteOBJ(const std::string& path) const {
    check(fs_write_obj(solver_.context(), path.c_str()), "fs_write_obj");
  }

 private:
  const EULERIAN_FLUID_SOLVER_3D& solver_;
};

inline std::vector<double> PROJECTION_3D::download(int field) const {
  std::vector<double> a((size_t)nx_ * ny_ * nz_);
  check(fs_download(ctx_, field, a.data(), nullptr), "fs_download");
  return a;
}

}  // namespace fluid_b200

#endif  // FLUID_B200_SOLVER_HPP
