"""Timestep benchmark: rising air bubble at 256^3 (density ratio 1000).

One "step" is one full timestep of the solver (fs_step: WENO5 TVD-RK3 level
set, three SolveForRK stages of WENO5 velocity advection + gravity +
semi-implicit viscosity + pressure projection, RK3 of reinitialisation
blocks) on the workload of the rising-bubble configuration: 256^3 cells on the
unit cube, air sphere of radius 0.15 at (0.5, 0.25, 0.5) (rho 1, mu 1.8e-5)
in water (rho 1000, mu 1e-3), gravity -9.8 y, CFL 0.5, pressure solved to
1e-6 relative divergence ||b - A p||/||b||.

`value` is the FP32+FP64-refinement timestep in ms (device time, inputs
resident).  The same steps are also timed in the plain FP64 path
(`fp64_ms_per_step`).  Inputs are synthetic (the scene above, seeded), the
fields are far larger than L2 (each FP32 field is 67 MB, a step touches
several GB), so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--n 256] [--impl reference]

With N > 1 (torchrun) every rank runs an independent replica of the same
workload on its own GPU ("replicas only": the path does not shard on one
GPU's worth of grid); `value` is then the max over ranks of the per-step time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# algorithmic bytes per unknown and PCG iteration (each array element once per pass)
# FP32+refine: spmv 20 (p, ax, ay, az read; q write) + residual update 14 (r, q read, bf16 1/diag read;
#              r write) + direction update 30 (x64 read/write, p read/write, r read, bf16 1/diag read)
BYTES_PER_UNKNOWN_PCG_FP32 = 64
# FP64: spmv 40 + residual update 32 + direction update 48
BYTES_PER_UNKNOWN_PCG_FP64 = 120
# red-black IC(0) (per cell of the grid, the black vectors holding half the
# cells): SpMV 16 (ax, ay, az 12; black p 2; black q 2) + residual update 7 +
# direction update 15, at about half the iterations
BYTES_PER_CELL_PCG_RB = 38
# DRAM bytes (read + write) of one FP32 Jacobi PCG iteration at 256^3
# measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum of
# k_cg_spmv, k_cg_update, k_cg_pupdate, one capture of the bench workload);
# scaled by the unknowns for other sizes
TRAFFIC_PER_ITERATION_256_FP32 = 1006.4e6
TRAFFIC_PER_ITERATION_256_RB = None


def scene(n):
    x = (np.arange(n) + 0.5) / n
    phi = np.sqrt((x[None, None, :] - 0.5) ** 2 + (x[None, :, None] - 0.25) ** 2 + (x[:, None, None] - 0.5) ** 2) - 0.15
    u = np.zeros((n, n, n + 1)); v = np.zeros((n, n + 1, n)); w = np.zeros((n + 1, n, n))
    return phi, u, v, w


PRECONDITIONER = {"default": 0, "jacobi": 1, "bf16": 2, "red_black": 3, "red_black_jacobi": 4}
PRECOND_CHOICE = "default"
# what FS_PRECOND_DEFAULT selects in an FP32_REFINE context
DEFAULT_FP32_PRECONDITIONER = "red_black"


def effective_preconditioner(fs):
    return DEFAULT_FP32_PRECONDITIONER if PRECOND_CHOICE == "default" else PRECOND_CHOICE
HOST_LOOP = 0  # 1: Krylov batches launched from the host (for profilers), not as one graph per solve


def params(fs, precision):
    pc = PRECONDITIONER[PRECOND_CHOICE] if precision == fs.FS_PRECISION_FP32_REFINE else 0
    return fs.default_params(pressure_preconditioner=pc, host_loop=HOST_LOOP,
                             rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, gravity=(0.0, -9.8, 0.0),
                             precision=precision, stop=fs.FS_STOP_RELATIVE, tolerance=1e-6, max_iteration=20000,
                             inner_tolerance=1e-3, max_outer=30, viscosity=1, viscosity_tolerance=1e-8, cfl=0.5,
                             order=3, reinit_iterations=10, reinit_scaling=5, weno_epsilon=1e-6)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in self.rows for q in range(4) if r[3 + q].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def run_steps(fs, n, precision, warmup, steps, barrier, record=0):
    """W untimed steps, then K steps timed by the library (CUDA events on its
    stream).  With record > 0 the state before each of the first `record`
    timed steps and its dt are kept in pinned host memory, so that the
    end-to-end run can replay exactly the same steps."""
    import torch
    phi, u, v, w = scene(n)
    s = fs.Solver(n, 1.0 / n, params(fs, precision))
    for k, a in zip(("phi", "u", "v", "w"), (phi, u, v, w)):
        s.upload(k, a)
    for _ in range(warmup):
        s.step(s.cfl_dt(), allow_not_converged=True)
    barrier()
    torch.cuda.synchronize()
    reps, states = [], []
    for m in range(steps):
        dt = s.cfl_dt()
        if m < record:
            states.append(({k: torch.from_numpy(s.download(k)).pin_memory() for k in ("phi", "u", "v", "w")}, dt))
        reps.append(s.step(dt, allow_not_converged=True))
    torch.cuda.synchronize()
    barrier()
    # divergence of the last projection's input (stored as div/dt), for the
    # relative divergence of the corrected velocity (outside the timed region)
    if reps:
        reps[-1]["div_input_l2"] = float(np.linalg.norm(s.download("divergence"))) * dt
    return s, reps, states


def e2e_steps(fs, s, states):
    """End to end through the public API, on the same steps as the timed run:
    per step, the state before it is uploaded from pinned host memory, the
    step runs with the same dt, and the level set is read back to pinned host
    memory.  Wall clock around the whole sequence, synchronised on both sides."""
    import torch
    shapes = {k: s.shape(k) for k in ("phi", "u", "v", "w")}
    out = torch.empty(shapes["phi"], dtype=torch.float64).pin_memory()
    h2d = sum(int(np.prod(sh)) * 8 for sh in shapes.values())
    d2h = int(np.prod(shapes["phi"])) * 8
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for host, dt in states:
        for k in ("phi", "u", "v", "w"):
            s.upload_ptr(k, host[k].data_ptr())
        s.step(dt, allow_not_converged=True)
        s.download_ptr("phi", out.data_ptr())
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3 / max(len(states), 1)
    return ms, h2d, d2h


def adjoint_steps(fs, n, warmup, steps, precision):
    """Adjoint step (fs_step_adjoint: forward recomputed with its tape, then
    the reverse sweep with the transposed solves) against the forward step
    from the same states in the same context, both timed by the library with
    CUDA events.  The bars are those of L = sum(phi^2) + |u|^2 at the step's
    end (any bar costs the same)."""
    s = fs.Solver(n, 1.0 / n, params(fs, precision))
    phi, u, v, w = scene(n)
    for k, a in zip(("phi", "u", "v", "w"), (phi, u, v, w)):
        s.upload(k, a)
    for _ in range(warmup):
        s.step(s.cfl_dt(), allow_not_converged=True)
    fwd, adj = [], []
    for _ in range(steps):
        dt = s.cfl_dt()
        st = {k: s.download(k) for k in ("phi", "u", "v", "w", "pressure")}
        fwd.append(s.step(dt, allow_not_converged=True)["ms"])
        bars = {k: 2.0 * s.download(k) for k in ("phi", "u", "v", "w")}
        for k, a in st.items():
            s.upload(k, a)
        s.adjoint_reset()
        for k, a in bars.items():
            s.upload("adj_" + k, a)
        adj.append(s.step_adjoint(dt, allow_not_converged=True)["ms"])
    mem = s.memory_bytes()
    s.close()
    f, a = float(np.mean(fwd)), float(np.mean(adj))
    return {"ms_per_step": a, "forward_ms_per_step": f, "ratio_to_forward": a / f, "steps": steps,
            "context_gib": mem / 2 ** 30}


class _TimedSolver:
    """The solver seen by the checkpoint schedules, keeping the library's
    device time of every forward and adjoint step."""

    def __init__(self, s):
        self.s, self.fwd, self.adj = s, [], []

    def step(self, dt):
        self.fwd.append(self.s.step(dt, allow_not_converged=True)["ms"])

    def step_adjoint(self, dt):
        self.adj.append(self.s.step_adjoint(dt, allow_not_converged=True)["ms"])

    def upload(self, k, a):
        self.s.upload(k, a)

    def download(self, k):
        return self.s.download(k)


def scene_params(fs, name, precision):
    if name == "dam_break":
        return fs.default_params(rho_neg=1000.0, rho_pos=1.0, mu_neg=1e-3, mu_pos=1.8e-5, gravity=(0.0, -9.8, 0.0),
                                 precision=precision, stop=fs.FS_STOP_RELATIVE, tolerance=1e-6, max_iteration=20000,
                                 viscosity=1, viscosity_tolerance=1e-8, cfl=0.5, order=3, reinit_iterations=10,
                                 reinit_scaling=5, host_loop=HOST_LOOP,
                                 pressure_preconditioner=(PRECONDITIONER[PRECOND_CHOICE]
                                                          if precision == fs.FS_PRECISION_FP32_REFINE else 0))
    if name == "rayleigh_taylor":
        return fs.default_params(rho_neg=850.0, rho_pos=1000.0, mu_neg=5e-2, mu_pos=1e-3, gravity=(0.0, -9.8, 0.0),
                                 precision=precision, stop=fs.FS_STOP_RELATIVE, tolerance=1e-6, max_iteration=40000,
                                 viscosity=1, viscosity_tolerance=1e-8, cfl=0.5, order=3, reinit_iterations=10,
                                 reinit_scaling=5, pressure_preconditioner=PRECONDITIONER[PRECOND_CHOICE],
                                 host_loop=HOST_LOOP)
    return params(fs, precision)


def run_scene(fs, name, steps, lead_in, window, snapshots):
    """The long configurations, one JSON line each (device times from the
    library's CUDA events; volumes with the reference's smeared Heaviside):

    - dam_break_128: 128^3 dam break, `steps` steps (default 200) in FP64
      and in FP32+refine from the same state at 1e-6 relative divergence;
      per-step time, PCG iterations, final divergence and the FP32+refine
      pressure and level set against the FP64 run's;
    - rising_bubble_256: `steps` steps (default 300) of the benchmark scene
      in FP32+refine with the bubble volume drift;
    - rayleigh_taylor_512_adjoint: 512^3 oil/water Rayleigh-Taylor with
      semi-implicit viscosity in FP32+refine, `lead_in` forward steps
      (default 84) then the gradient of L = ||phi(T)||^2 over the last
      `window` steps (default 16) with binomial checkpointing (`snapshots`
      snapshots, default 3), with the context's and the device's memory."""
    import torch

    from fluid_simulator_backup_b200 import checkpoint as ck
    from fluid_simulator_backup_b200 import scenes as sc
    out = {"scene": name}
    if name == "dam_break_128":
        n = 128
        steps = steps or 200
        phi0 = sc.dam_break(n)
        v0 = sc.heaviside_volume(phi0, 1.0 / n)
        res = {}
        for prec, key in ((fs.FS_PRECISION_FP64, "fp64"), (fs.FS_PRECISION_FP32_REFINE, "fp32_refine")):
            with fs.Solver(n, 1.0 / n, scene_params(fs, "dam_break", prec)) as s:
                s.upload("phi", phi0)
                for k, a in zip("uvw", sc.zero_faces(n)):
                    s.upload(k, a)
                reps = [s.step(s.cfl_dt(), allow_not_converged=True) for _ in range(steps)]
                phi, p = s.download("phi"), s.download("pressure")
            res[key] = (phi, p - p.mean())
            out[key] = {"ms_per_step": float(np.mean([r["ms"] for r in reps])),
                        "pcg_iterations_per_step": float(np.mean([r["pcg_iterations"] for r in reps])),
                        "max_rel_residual": max(r["max_rel_residual"] for r in reps),
                        "div_l2_final": reps[-1]["div_l2"], "div_linf_final": reps[-1]["div_linf"],
                        "div_linf_max": max(r["div_linf"] for r in reps),
                        "volume_drift": sc.heaviside_volume(phi, 1.0 / n) / v0 - 1}
        (phi64, p64), (phi32, p32) = res["fp64"], res["fp32_refine"]
        out.update(grid=[n] * 3, steps=steps, speedup_fp32_refine=out["fp64"]["ms_per_step"] /
                   out["fp32_refine"]["ms_per_step"],
                   pressure_rel_diff=float(np.linalg.norm(p32 - p64) / np.linalg.norm(p64)),
                   phi_max_diff=float(np.abs(phi32 - phi64).max()))
    elif name == "rising_bubble_256":
        n = 256
        steps = steps or 300
        phi0 = sc.rising_bubble(n)
        v0 = sc.heaviside_volume(phi0, 1.0 / n)
        with fs.Solver(n, 1.0 / n, params(fs, fs.FS_PRECISION_FP32_REFINE)) as s:
            s.upload("phi", phi0)
            for k, a in zip("uvw", sc.zero_faces(n)):
                s.upload(k, a)
            reps, t = [], 0.0
            for _ in range(steps):
                dt = s.cfl_dt()
                reps.append(s.step(dt, allow_not_converged=True))
                t += dt
            phi = s.download("phi")
        out.update(grid=[n] * 3, steps=steps, simulated_time=t,
                   ms_per_step=float(np.mean([r["ms"] for r in reps])),
                   pcg_iterations_per_step=float(np.mean([r["pcg_iterations"] for r in reps])),
                   max_rel_residual=max(r["max_rel_residual"] for r in reps),
                   div_l2_final=reps[-1]["div_l2"], div_linf_max=max(r["div_linf"] for r in reps),
                   bubble_volume_drift=sc.heaviside_volume(phi, 1.0 / n) / v0 - 1)
    elif name == "rayleigh_taylor_512_adjoint":
        n = 512
        lead_in = 84 if lead_in is None else lead_in
        free0, total = torch.cuda.mem_get_info()
        with fs.Solver(n, 1.0 / n, scene_params(fs, "rayleigh_taylor", fs.FS_PRECISION_FP32_REFINE)) as s:
            s.upload("phi", sc.rayleigh_taylor(n))
            for k, a in zip("uvw", sc.zero_faces(n)):
                s.upload(k, a)
            dt = s.cfl_dt()  # one dt for the whole run, so that the window is one differentiable map
            lead = [s.step(dt, allow_not_converged=True)["ms"] for _ in range(lead_in)]
            st0 = ck.save(s)
            ts, sched = _TimedSolver(s), ck.Schedule()
            t0 = time.perf_counter()
            end = ck.advance(ts, st0, window, dt, sched)
            t_fwd = time.perf_counter() - t0
            s.adjoint_reset()
            for k in ck.KEYS:
                s.upload("adj_" + k, 2.0 * end[k] if k == "phi" else np.zeros_like(end[k]))
            t0 = time.perf_counter()
            ck.reverse_binomial(ts, 0, window, st0, snapshots, dt, sched)
            t_rev = time.perf_counter() - t0
            free1, _ = torch.cuda.mem_get_info()
            ctx_bytes = s.memory_bytes()
            bars = {k: s.download("adj_" + k) for k in ck.KEYS}
            rho_bar = s.density_bars()[0]
        fwd_ms = float(np.mean(ts.fwd))
        adj_ms = float(np.mean(ts.adj))
        out.update(grid=[n] * 3, dt=dt, lead_in_steps=lead_in, window_steps=window, snapshots=snapshots,
                   lead_in_ms_per_step=float(np.mean(lead)) if lead else None,
                   window_forward_ms_per_step=fwd_ms, adjoint_ms_per_step=adj_ms, adjoint_to_forward=adj_ms / fwd_ms,
                   forward_steps_in_reversal=sched.forward_steps - window, adjoint_steps=sched.adjoint_steps,
                   max_live_snapshots=sched.max_live_snapshots, window_forward_wall_s=t_fwd,
                   reversal_wall_s=t_rev, context_gib=ctx_bytes / 2 ** 30,
                   device_in_use_gib=(total - free1) / 2 ** 30, device_total_gib=total / 2 ** 30,
                   device_in_use_before_gib=(total - free0) / 2 ** 30,
                   bars_finite=bool(all(np.isfinite(b).all() for b in bars.values())),
                   d_loss_d_rho_oil=rho_bar)
    else:
        raise ValueError(name)
    return out


def reference_tolerance(m, rel=1e-6):
    """The reference's PCG stops on an absolute test, r.z < tol^2
    (PCG_METHOD.cpp:87).  The tolerance that matches the GPU path's relative
    test ||r||/||b|| <= rel on the scene's first projection: rel times
    sqrt(b.D^-1 b) of that system.  The first stage projects u* = (0, g dt,
    0) on interior faces (zero walls), so b = div(g) does not depend on dt."""
    from oracle import fs_oracle as O
    phi, u, v, w = scene(m)
    dt = 1.0
    v = v.copy()
    v[:, 1:-1, :] = -9.8 * dt
    b = -O.divergence(u, v, w, 1.0 / m, dt)
    b = b - b.mean()
    diag = O.poisson_operator(phi, 1.0 / m, 1.0, 1000.0)[3]
    return rel * float(np.sqrt(np.sum(b * b / diag)))


def reference_frames(sizes, frames, budget_s, lib_name="libfsref.so"):
    """Whole reference timesteps, timed on the host: for each sample grid m
    the rising-bubble scene is injected into the reference's own solver
    (oracle/_ref, built from the reference sources) and
    SIMULATION_WORLD::AdvanceOneFrame (SIMULATION_WORLD.h:320) runs one
    untimed frame, then up to `frames` timed frames within budget_s seconds:
    dt from the reference's CFL condition, three RK stages of WENO5 velocity
    advection, gravity, its air/water viscosity and a projection whose PCG
    runs to convergence, WENO5 level set and Sussman reinitialisation, all
    in the reference's FP64 code on one thread.  Runs in a child process
    (the reference calls exit() on some inputs and holds ~2.3 kB of host
    memory per cell).  Returns {m: {"ms": [...], "pcg_iterations": [...]}}."""
    code = ("import json, sys; sys.path.insert(0, %r); import bench; "
            "print('REFJSON' + json.dumps(bench._reference_frames_here(%r, %d, %r)))"
            % (ROOT, list(sizes), frames, float(budget_s)))
    env = dict(os.environ, FSREF_LIB=lib_name)
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, timeout=1800, env=env)
    for line in p.stdout.splitlines():
        if line.startswith("REFJSON"):
            return {int(k): v for k, v in json.loads(line[7:]).items()}
    raise RuntimeError(f"reference frames failed (rc={p.returncode}): {p.stderr.strip()[-300:]}")


def _reference_frames_here(sizes, frames, budget_s):
    import shutil
    import tempfile

    from oracle import refsim
    if not refsim.available():
        raise RuntimeError("oracle/_ref is not built")
    out = {}
    tmp = tempfile.mkdtemp(prefix="fs_ref_")
    try:
        for m in sizes:
            # the iteration cap: 40 m, far above the converged counts (115-286
            # at 32^3-64^3); a later frame whose system stagnates above the
            # matched absolute tolerance stops there instead of running for
            # minutes, and shows as the cap in the reported iteration counts
            path = refsim.write_sim(os.path.join(tmp, f"ref_{m}.sim"), m, water_drop=False, threads=1,
                                    tolerance=reference_tolerance(m), max_iteration=40 * m)
            c = refsim.RefCase(path)
            phi, u, v, w = scene(m)
            for k, a in zip(("phi", "u", "v", "w"), (phi, u, v, w)):
                c.set(k, a)
            c.advance_frame()  # untimed
            ms, its = [], []
            t_start = time.perf_counter()
            while len(ms) < frames and (not ms or time.perf_counter() - t_start < budget_s / len(sizes)):
                t = time.perf_counter()
                _, it = c.advance_frame()
                ms.append((time.perf_counter() - t) * 1e3)
                its.append(it)
            c.close()
            out[m] = {"ms": ms, "pcg_iterations": its}
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return out


def reference_estimate(n, sizes, frames, budget_s):
    """The reference's step time at n^3 from whole reference frames at two
    sample grids.  Per frame the reference does work proportional to the
    cells (advection, viscosity, reinitialisation, system build) plus its
    Jacobi-PCG, whose iteration count grows about linearly with n (186-226
    at 48^3, 274-286 at 64^3 on this scene).  The estimate is the larger
    grid's mean frame scaled by the cell count, (n/m)^3: a lower bound of
    the reference's time at n^3, since it leaves out the growth of the PCG
    iterations.  The fit t(m) = a m^3 + b m^4 through both means, which
    would include it, is reported beside it: two close grids with timing
    noise of a few per cent move that fit by a factor of two."""
    import platform
    res = reference_frames(sizes, frames, budget_s)
    (m1, m2) = sizes
    t1, t2 = float(np.mean(res[m1]["ms"])), float(np.mean(res[m2]["ms"]))
    A = np.array([[m1 ** 3, m1 ** 4], [m2 ** 3, m2 ** 4]], dtype=float)
    a, b = np.linalg.solve(A, np.array([t1, t2]))
    est = t2 * (n / m2) ** 3
    fit = f"{(a * n ** 3 + b * n ** 4) / 1e3:.0f} s" if a >= 0 and b >= 0 else "not positive"
    model = (f"t({m2}) x ({n}/{m2})^3, a lower bound (the m^3 + m^4 fit through both grids, which counts the "
             f"growth of the PCG iterations: {fit})")
    try:
        cpu_model = next(l.split(":", 1)[1].strip() for l in open("/proc/cpuinfo") if l.startswith("model name"))
    except Exception:
        cpu_model = platform.processor() or "unknown"
    frames_run = {m: len(res[m]["ms"]) for m in sizes}
    sample = (f"whole reference frames (SIMULATION_WORLD::AdvanceOneFrame, FP64, PCG to an absolute tolerance "
              f"matching 1e-6 relative on the first projection), 1 thread (with more threads a whole frame of the "
              f"headless build does not finish); one untimed frame then {frames_run[m1]} timed at {m1}^3 "
              f"(mean {t1:.0f} ms, PCG iterations {res[m1]['pcg_iterations']}) and {frames_run[m2]} timed at "
              f"{m2}^3 (mean {t2:.0f} ms, PCG iterations {res[m2]['pcg_iterations']}); scaled to {n}^3 by {model}; "
              f"host: {os.cpu_count()} logical cores, {cpu_model}")
    return est, sample, frames_run


def init_replicas(backend="nccl"):
    """One process per GPU, each running an independent replica of the
    workload ("replicas only": the path has no exchange step).  Returns the
    rank layout, the process group module (None for one process) and the two
    collectives the benchmark uses: a barrier around the timed region and the
    max over ranks of a per-rank time.  With backend "gloo" everything stays
    on the CPU (used by the multi-process tests)."""
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    device = "cpu" if backend == "gloo" else "cuda"
    if world > 1:
        import datetime

        import torch.distributed as dist
        if device == "cuda":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    elif device == "cuda":
        torch.cuda.set_device(0)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    return world, rank, local, dist, barrier, max_over_ranks


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--precision", default="fp32_refine", choices=["fp32_refine", "fp64"],
                    help="precision of the timed path (the headline is fp32_refine)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward measurement")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--preconditioner", default="default", choices=sorted(PRECONDITIONER),
                    help="pressure preconditioner of the FP32+refine path (the FP64 comparison stays Jacobi)")
    ap.add_argument("--host-loop", action="store_true",
                    help="launch the Krylov batches from the host instead of one graph per solve (for ncu)")
    ap.add_argument("--scene", default=None,
                    choices=["dam_break_128", "rising_bubble_256", "rayleigh_taylor_512_adjoint"],
                    help="run one of the long configurations instead of the timestep benchmark (1 GPU)")
    ap.add_argument("--scene-steps", type=int, default=None)
    ap.add_argument("--lead-in", type=int, default=None)
    ap.add_argument("--window", type=int, default=16)
    ap.add_argument("--snapshots", type=int, default=3)
    args = ap.parse_args()
    global PRECOND_CHOICE, HOST_LOOP
    PRECOND_CHOICE = args.preconditioner
    HOST_LOOP = 1 if args.host_loop else 0

    # the reference arm is host work: its ranks meet over gloo and touch no GPU
    world, rank, local, dist, barrier, max_over_ranks = init_replicas("gloo" if args.impl == "reference" else "nccl")

    n = args.n
    config = {"workload": f"rising air bubble {n}^3, density ratio 1000, one timestep (TVD-RK3, 3 projections)",
              "grid": [n, n, n], "precision": "fp32+fp64-refine", "div_tolerance": 1e-6, "cfl": 0.5,
              "l2": "inputs larger than L2 (67 MB per FP32 field), no flush", "parallelism": f"replicas{world}"}
    metric = "timestep ms @256^3 (FP32+refine, 1e-6 relative divergence); adjoint/fwd ratio in adjoint"

    if args.impl == "reference":
        if rank != 0:
            if dist is not None:
                dist.destroy_process_group()
            return
        # whole reference frames at 48^3 and 64^3 (about a minute on one host
        # thread), scaled to n^3; the steps printed are the frames run.  At
        # 32^3 the reference's PCG stalls above the matched tolerance after
        # the first frame (every later frame ends at the iteration cap), so
        # that grid says nothing about the reference's converged frame.
        ms, sample, frames_run = reference_estimate(n, (48, 64), frames=max(1, args.steps), budget_s=120.0)
        steps_run = sum(frames_run.values())
        line = {"impl": "reference", "metric": metric, "value": ms, "unit": "ms", "n_gpus": args.gpus,
                "steps": steps_run, "warmup": len(frames_run), "ms_per_step": ms, "higher_is_better": False,
                "dtype": "f64", "data": "synthetic", "config": config,
                "steps_note": "timed reference frames per sample grid %s after one untimed frame each" % frames_run,
                "cpu_baseline": {"value": ms, "unit": "ms", "cores": 1, "kind": "reference", "sample": sample,
                                 "host_cores": os.cpu_count()},
                "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        if dist is not None:
            dist.destroy_process_group()
        return

    import fluid_simulator_backup_b200 as fs
    fs.lib()
    if args.scene:
        with ClockSampler(local) as clk:
            out = run_scene(fs, args.scene, args.scene_steps, args.lead_in, args.window, args.snapshots)
        out.update(preconditioner=PRECOND_CHOICE, clocks=clk.summary())
        if rank == 0:
            print(json.dumps(out))
        if dist is not None:
            dist.destroy_process_group()
        return
    main_prec = fs.FS_PRECISION_FP32_REFINE if args.precision == "fp32_refine" else fs.FS_PRECISION_FP64
    if main_prec == fs.FS_PRECISION_FP64:
        args.no_fp64 = True
        config["precision"] = "fp64"
    with ClockSampler(local) as clk:
        s32, reps, states = run_steps(fs, n, main_prec, args.warmup, args.steps, barrier,
                                      record=min(args.e2e_steps, args.steps))
    ms_steps = [r["ms"] for r in reps]
    ms = max_over_ranks(float(np.mean(ms_steps)))
    pcg_ms = sum(r["pcg_ms"] for r in reps)
    pcg_its = sum(r["pcg_launched_iterations"] for r in reps)
    real_its = sum(r["pcg_iterations"] for r in reps)
    launches = sum(r["kernel_launches"] for r in reps)
    N = n ** 3
    # device time of the pressure solves per real iteration (the launched
    # count adds the idle tail of the last graph batch of each solve)
    per_iter_s = pcg_ms / 1e3 / max(real_its, 1)
    rb = main_prec == fs.FS_PRECISION_FP32_REFINE and effective_preconditioner(fs) in ("red_black", "red_black_jacobi")
    if main_prec == fs.FS_PRECISION_FP64:
        bpu, kernel = BYTES_PER_UNKNOWN_PCG_FP64, "FP64 Jacobi PCG iteration (spmv + update + direction, 3 kernels)"
        traffic = None
    elif rb:
        bpu = BYTES_PER_CELL_PCG_RB
        kernel = ("red-black IC(0) PCG iteration (Schur-complement red and black passes, p.q, residual update, "
                  "direction update: 5 kernels)")
        traffic = TRAFFIC_PER_ITERATION_256_RB * N / 256 ** 3 if TRAFFIC_PER_ITERATION_256_RB else None
    else:
        bpu, kernel = BYTES_PER_UNKNOWN_PCG_FP32, "FP32 Jacobi PCG iteration (spmv + update + direction, 3 kernels)"
        traffic = TRAFFIC_PER_ITERATION_256_FP32 * N / 256 ** 3
    achieved = bpu * N / per_iter_s / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    e2e_ms, h2d, d2h = e2e_steps(fs, s32, states)
    e2e_ms = max_over_ranks(e2e_ms)
    # the device time of the same steps, for comparison with the end-to-end figure
    e2e_device_ms = float(np.mean([r["ms"] for r in reps[:len(states)]])) if states else None
    del states
    s32.close()

    fp64 = None
    if not args.no_fp64:
        s64, reps64, _ = run_steps(fs, n, fs.FS_PRECISION_FP64, args.warmup, args.steps, barrier)
        ms64 = max_over_ranks(float(np.mean([r["ms"] for r in reps64])))
        fp64 = {"ms_per_step": ms64, "pcg_iterations_per_step": float(np.mean([r["pcg_iterations"] for r in reps64])),
                "speedup_fp32_refine": ms64 / ms, "max_rel_residual": max(r["max_rel_residual"] for r in reps64)}
        s64.close()

    adjoint = None
    if not args.no_adjoint:
        adjoint = {}
        for prec, key in ((fs.FS_PRECISION_FP64, "fp64"), (fs.FS_PRECISION_FP32_REFINE, "fp32_refine")):
            a = adjoint_steps(fs, n, min(args.warmup, 1), min(args.steps, 2), prec)
            a["ms_per_step"] = max_over_ranks(a["ms_per_step"])
            adjoint[key] = a

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # bounded sample (about 20 s of host work): whole frames at 48^3 and 64^3
        try:
            ref_ms, sample, _ = reference_estimate(n, (48, 64), frames=2, budget_s=40.0)
            cpu = {"value": ref_ms, "unit": "ms", "cores": 1, "kind": "reference", "sample": sample,
                   "host_cores": os.cpu_count()}
        except Exception as e:  # the baseline is reported, not required
            cpu = {"value": None, "unit": "ms", "cores": 1, "kind": "reference", "sample": f"failed: {e}"}

    line = {
        "metric": metric, "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if main_prec == fs.FS_PRECISION_FP32_REFINE else "f64",
        "data": "synthetic", "config": config,
        "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": "the first %d timed steps replayed from their saved states" % min(args.e2e_steps, args.steps),
                "device_ms_same_steps": e2e_device_ms},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": kernel, "preconditioner": effective_preconditioner(fs),
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_src,
                     "traffic": traffic,
                     "traffic_unit": "bytes per PCG iteration (ncu capture at 256^3, scaled by unknowns)",
                     "bytes_per_iteration": bpu * N,
                     "pcg_ms": pcg_ms, "pcg_launched_iterations": pcg_its, "pcg_iterations": real_its},
        "fp64": fp64,
        "adjoint": adjoint,
        "divergence": {"div_l2_last": reps[-1]["div_l2"], "div_linf_max": max(r["div_linf"] for r in reps),
                       "div_input_l2_last": reps[-1].get("div_input_l2"),
                       "relative_l2_last": (reps[-1]["div_l2"] / reps[-1]["div_input_l2"]
                                            if reps[-1].get("div_input_l2") else None),
                       "max_rel_residual": max(r["max_rel_residual"] for r in reps)},
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    if rank == 0:
        # per-step detail on stderr; the one JSON line on stdout stays short
        detail = [{k: r[k] for k in ("ms", "pcg_iterations", "outer_iterations", "viscosity_iterations",
                                     "max_rel_residual", "div_l2", "div_linf", "pcg_ms")} for r in reps]
        print(json.dumps({"steps_detail": detail}), file=sys.stderr)
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
