// Test driver for include/fluid_b200_solver.hpp (built and run by
// tests/test_cpp_mirror.py).  Modes:
//   script <file.sim>               parse a script, print a few values
//   csr <problem.bin> <out.bin>     CUDA_PCG_METHOD on a CSR system
//   step <file.sim> <phi.bin> <out.bin>
//                                   one AdvanceOneTimeStepThread from phi and zero velocity
// Binary files are raw little-endian values (see the Python side).
#include <cstdio>
#include <fstream>
#include <iostream>
#include <vector>

#include "fluid_b200_solver.hpp"

using namespace fluid_b200;

template <class T>
static std::vector<T> read_vec(std::ifstream& f, size_t n) {
  std::vector<T> v(n);
  f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(T)));
  return v;
}

template <class T>
static void write_vec(std::ofstream& f, const std::vector<T>& v) {
  f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const std::string mode = argv[1];
  try {
    if (mode == "script") {
      SCRIPT_READER r(argv[2]);
      const SCRIPT_BLOCK& world = r.FindBlock("SIMULATION_WORLD");
      GRID_STRUCTURE_3D g;
      g.InitializeFromBlock(world.FindBlock("WORLD_DISCRETIZATION_AIR_WATER").FindBlock("GRID_STRUCTURE_3D_LARGE"));
      const fs_params p = params_from_block(r.FindBlock("FLUID_SOLVER_UNIFORM_AIR_WATER"), g);
      std::printf("res %d %d %d dx %.17g\n", g.i_res, g.j_res, g.k_res, g.dx);
      std::printf("rho %.17g %.17g mu %.17g %.17g\n", p.rho_neg, p.rho_pos, p.mu_neg, p.mu_pos);
      std::printf("tol %.17g maxit %d stop %d order %d reinit %d %d cfl %.17g\n", p.tolerance, p.max_iteration,
                  p.stop, p.order, p.reinit_iterations, p.reinit_scaling, world.GetFloat("CFL", 0.5));
      std::printf("velocity_scheme %d velocity_epsilon %.17g\n", p.velocity_scheme, p.velocity_epsilon);
      std::printf("fast_sweeping %d reinit_iterations %d\n", p.fast_sweeping, p.reinit_iterations);
      return 0;
    }
    if (mode == "pipe_script") {
      // the pipe reader's parameters (no GPU needed)
      SCRIPT_READER r(argv[2]);
      const SCRIPT_BLOCK& world = r.FindBlock("SIMULATION_WORLD");
      const SCRIPT_BLOCK& disc = world.FindBlock("WORLD_DISCRETIZATION_OIL_WATER");
      GRID_STRUCTURE_3D g;
      g.InitializeFromBlock(disc.FindBlock("GRID_STRUCTURE_3D_VERTICAL"));
      const fs_params p = pipe_params_from_script(world, r.FindBlock("FLUID_SOLVER_UNIFORM_OIL_WATER"), g);
      std::printf("pipe %d radius %.17g R1 %.17g V0 %.17g f %.17g eta %.17g We %.17g oil %.17g rho_pos %.17g "
                  "order %d viscosity %d cfl %.17g\n",
                  p.pipe, p.pipe_radius, p.pipe_R1, p.pipe_V0, p.pipe_f, p.pipe_eta, p.pipe_We, p.pipe_oil_density,
                  p.rho_pos, p.order, p.viscosity, p.cfl);
      return 0;
    }
    if (mode == "csr" && argc >= 4) {
      std::ifstream f(argv[2], std::ios::binary);
      int hdr[2];
      double tol;
      int maxit;
      f.read(reinterpret_cast<char*>(hdr), sizeof hdr);
      f.read(reinterpret_cast<char*>(&tol), sizeof tol);
      f.read(reinterpret_cast<char*>(&maxit), sizeof maxit);
      CSR_MATRIX<double> A;
      A.N = hdr[0];
      A.nz = hdr[1];
      A.values = read_vec<double>(f, A.nz);
      A.column_index = read_vec<int>(f, A.nz);
      A.row_ptr = read_vec<int>(f, A.N + 1);
      VECTOR_ND<double> b, x(A.N, 0.0);
      b.values = read_vec<double>(f, A.N);
      b.num_dimension = A.N;
      FIELD_STRUCTURE_3D<int> bc;  // the boundary tags the reference passes along
      CUDA_PCG_METHOD solver;
      LINEAR_SOLVER& ls = solver;  // through the plugin base, as POISSON_SOLVER_3D holds it
      ls.Initialize(tol, maxit);
      for (int t = 3; t >= 0; --t) ls.Solve(t, A, x, b, bc);  // worker threads 1..3 return at once
      std::ofstream o(argv[3], std::ios::binary);
      write_vec(o, x.values);
      std::printf("iterations %d residual %.17g\n", ls.num_iteration, ls.residual);
      return 0;
    }
    if (mode == "step" && argc >= 5) {
      EULERIAN_FLUID_SOLVER_3D s;
      s.InitializeFromScript(argv[2]);
      std::ifstream f(argv[3], std::ios::binary);
      s.SetField(FS_FIELD_PHI, read_vec<double>(f, (size_t)s.Count(FS_FIELD_PHI)));
      for (int fld : {FS_FIELD_U, FS_FIELD_V, FS_FIELD_W}) s.SetField(fld, std::vector<double>((size_t)s.Count(fld), 0.0));
      const double dt = s.CFL() * s.CFLOneTimeStep();
      s.AdvanceOneTimeStepThread(1, dt);  // not the head thread: no work
      s.AdvanceOneTimeStepThread(0, dt);
      s.water_projection->Solve(2, dt);
      std::ofstream o(argv[4], std::ios::binary);
      write_vec(o, s.GetField(FS_FIELD_PHI));
      std::printf("dt %.17g pcg %d status %d\n", dt, s.last_report.pcg_iterations, (int)s.last_status);
      return 0;
    }
    if (mode == "levelset" && argc >= 6) {
      // levelset <sim> <phi.bin> <phi_out.bin> <surface.obj>: the reference's
      // full fast sweeping, then the OBJ writer
      EULERIAN_FLUID_SOLVER_3D s;
      s.InitializeFromScript(argv[2]);
      std::ifstream f(argv[3], std::ios::binary);
      s.SetField(FS_FIELD_PHI, read_vec<double>(f, (size_t)s.Count(FS_FIELD_PHI)));
      s.FullFastSweepingMethodThreaded();
      s.ReinitializeByFastSweeping(1);  // not the head thread: no work
      std::ofstream o(argv[4], std::ios::binary);
      write_vec(o, s.GetField(FS_FIELD_PHI));
      WRITE_LEVELSET(s).WriteOBJ(argv[5]);
      std::printf("ok\n");
      return 0;
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 2;
}
