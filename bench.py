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
# DRAM bytes (read + write) of one FP32 PCG iteration at 256^3 measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum of k_cg_spmv, k_cg_update,
# k_cg_pupdate, one capture of the bench workload); scaled by the unknowns
# for other sizes
TRAFFIC_PER_ITERATION_256_FP32 = 1006.4e6
# PCG iterations per projection of the FP64 GPU path on this workload at 256^3
# (6725 per timestep of 3 projections over steps 4-6, measured by the default
# run's fp64 block); the reference arm prices its projection with it
REF_PCG_ITERATIONS_256 = 2242


def scene(n):
    x = (np.arange(n) + 0.5) / n
    phi = np.sqrt((x[None, None, :] - 0.5) ** 2 + (x[None, :, None] - 0.25) ** 2 + (x[:, None, None] - 0.5) ** 2) - 0.15
    u = np.zeros((n, n, n + 1)); v = np.zeros((n, n + 1, n)); w = np.zeros((n + 1, n, n))
    return phi, u, v, w


def params(fs, precision):
    return fs.default_params(rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, gravity=(0.0, -9.8, 0.0),
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


def adjoint_steps(fs, n, warmup, steps):
    """FP64 adjoint step (fs_step_adjoint: forward recomputed with its tape,
    then the reverse sweep with the transposed solves) against the FP64
    forward step from the same states, both timed by the library with CUDA
    events.  The bars are those of L = sum(phi^2) + |u|^2 at the step's end
    (any bar costs the same)."""
    s = fs.Solver(n, 1.0 / n, params(fs, fs.FS_PRECISION_FP64))
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
    s.close()
    f, a = float(np.mean(fwd)), float(np.mean(adj))
    return {"ms_per_step": a, "forward_fp64_ms_per_step": f, "ratio_to_forward": a / f, "precision": "fp64",
            "steps": steps}


def reference_sample(n, pcg_iterations_per_projection, threads=1):
    """Time the reference's own CPU operators (oracle/_ref, built from the
    reference sources) on the same 256^3 scene and scale them to one
    timestep: 3 level-set WENO5 updates, 3 WENO5 velocity updates, 3
    explicit viscosity updates (the reference's air/water viscosity), 3
    projections (system build + the GPU FP64 path's PCG iteration count per
    projection at the same tolerance) and 3 reinitialisation blocks of 10
    pseudo-steps.  Bounded sample: one call of each operator, the projection
    run at two iteration caps to separate build and per-iteration cost, one
    Sussman pseudo-step."""
    import psutil

    from oracle import refsim
    if not refsim.available():
        return None, "oracle/_ref/libfsref.so not built"
    # the reference holds ~150 double fields of n^3; sample at a smaller grid
    # and scale per cell when the host cannot hold the full one comfortably
    need_gb = 2300 * n ** 3 / 1e9  # ~2.3 kB of host memory per cell (measured at 64^3)
    # at most 128^3 (a bounded sample: per-cell costs scale to n^3; a smaller
    # grid caches better, so the scaled time errs in the reference's favour)
    m = min(n, 128)
    while need_gb * (m / n) ** 3 > 0.5 * psutil.virtual_memory().available / 1e9 and m > 64:
        m //= 2
    scale = (n / m) ** 3
    os.makedirs(os.path.join(ROOT, "_bench_tmp"), exist_ok=True)
    phi, u, v, w = scene(m)
    rng = np.random.default_rng(0)
    u = rng.normal(size=u.shape) * 0.01; v = rng.normal(size=v.shape) * 0.01; w = rng.normal(size=w.shape) * 0.01
    times = {}

    def case(max_iteration, reinit_iterations=1):
        path = refsim.write_sim(os.path.join(ROOT, "_bench_tmp", f"ref_{m}.sim"), m, water_drop=False, threads=threads,
                                tolerance=1e-30, max_iteration=max_iteration, reinit_iterations=reinit_iterations)
        c = refsim.RefCase(path)
        for k, a in zip(("phi", "u", "v", "w"), (phi, u, v, w)):
            c.set(k, a)
        return c

    c = case(5)
    t = time.perf_counter(); c.weno5_levelset(1e-4); times["weno_levelset"] = time.perf_counter() - t
    t = time.perf_counter(); c.weno5_velocity(1e-4, 1); times["weno_velocity"] = time.perf_counter() - t
    t = time.perf_counter(); c.viscosity(1e-4); times["viscosity"] = time.perf_counter() - t
    for k, a in zip(("phi", "u", "v", "w"), (phi, u, v, w)):
        c.set(k, a)
    t = time.perf_counter(); c.projection(1e-4); t5 = time.perf_counter() - t
    t = time.perf_counter(); c.reinitialization(1e-4, 0); times["reinit_pseudo_step"] = time.perf_counter() - t
    c.close()
    c = case(15)
    t = time.perf_counter(); c.projection(1e-4); t15 = time.perf_counter() - t
    c.close()
    per_it = max((t15 - t5) / 10.0, 0.0)
    build = max(t5 - 5 * per_it, 0.0)
    for f in os.listdir(os.path.join(ROOT, "_bench_tmp")):
        os.remove(os.path.join(ROOT, "_bench_tmp", f))
    os.rmdir(os.path.join(ROOT, "_bench_tmp"))
    step_s = scale * (3 * times["weno_levelset"] + 3 * times["weno_velocity"] + 3 * times["viscosity"] +
                      3 * (build + pcg_iterations_per_projection * per_it) + 3 * 10 * times["reinit_pseudo_step"])
    sample = (f"reference operators on {threads} thread(s), timed once each at {m}^3 (cells scale x{scale:g} to {n}^3): WENO5 level set "
              f"{times['weno_levelset']:.2f}s, WENO5 u,v,w {times['weno_velocity']:.2f}s, explicit viscosity "
              f"{times['viscosity']:.2f}s, projection build {build:.2f}s + {per_it * 1e3:.1f} ms/PCG iteration, "
              f"Sussman pseudo-step {times['reinit_pseudo_step']:.2f}s; scaled to 3 stages with "
              f"{pcg_iterations_per_projection:.0f} PCG iterations per projection and 3x10 pseudo-steps")
    return step_s * 1e3, sample


# builds of the reference sources tried for the CPU baseline: the one the
# goldens come from, and -O3 for x86-64-v3 (AVX2, FMA)
REF_BUILDS = (("-O2", "libfsref.so"), ("-O3 -march=x86-64-v3", "libfsref_o3.so"))


def reference_sample_best(n, iters):
    """The reference's operators on 1, 2, 4 ... up to every host core (its
    own MULTITHREADING domain decomposition), from each available build;
    the fastest is the baseline."""
    cores = os.cpu_count() or 1
    cands = sorted({t for t in (1, 2, 4, 8, 16, 32, cores) if t <= cores})
    best = (None, "reference sample failed", 1)
    tried = []
    for flags, name in REF_BUILDS:
        if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", name)):
            continue
        for t in cands:
            ms, sample = reference_sample_isolated(n, iters, t, name)
            if ms is None:
                tried.append(f"{flags} {t}: failed")
                continue
            tried.append(f"{flags} {t}: {ms / 1e3:.0f} s")
            if best[0] is None or ms < best[0]:
                best = (ms, f"build {flags}: " + sample, t)
    ms, sample, t = best
    return ms, (sample + "; step estimate per build and thread count: " + ", ".join(tried)), t


def reference_sample_isolated(n, iters, threads=1, lib="libfsref.so"):
    """reference_sample in a child process: the reference calls exit() on
    some inputs (LEVELSET_3D.h:1040-1044) and holds tens of GB of host
    memory at 256^3; neither should touch the benchmark process (nor an
    instruction the host lacks, for the x86-64-v3 build)."""
    code = ("import json, sys; sys.path.insert(0, %r); import bench; "
            "ms, sample = bench.reference_sample(%d, %r, %d); print('REFJSON' + json.dumps([ms, sample]))"
            % (ROOT, n, float(iters), threads))
    env = dict(os.environ, FSREF_LIB=lib)
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, timeout=1200, env=env)
    for line in p.stdout.splitlines():
        if line.startswith("REFJSON"):
            return tuple(json.loads(line[7:]))
    return None, f"reference sample failed (rc={p.returncode}): {p.stderr.strip()[-300:]}"


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
    args = ap.parse_args()

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
        # the FP64 PCG iteration count of this workload on the GPU path at the
        # same tolerance (measured in the default run; see profiles/)
        # (Jacobi-PCG iteration counts grow about linearly with n)
        iters = float(os.environ.get("FS_REF_PCG_ITERATIONS", str(REF_PCG_ITERATIONS_256 * n / 256.0)))
        ms, sample, threads = reference_sample_best(n, iters)
        line = {"impl": "reference", "metric": metric, "value": ms, "unit": "ms", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
                "dtype": "f64", "data": "synthetic", "config": config,
                "cpu_baseline": {"value": ms, "unit": "ms", "cores": threads, "kind": "reference", "sample": sample},
                "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        if dist is not None:
            dist.destroy_process_group()
        return

    import fluid_simulator_backup_b200 as fs
    fs.lib()
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
    per_iter_s = pcg_ms / 1e3 / max(pcg_its, 1)
    bpu = BYTES_PER_UNKNOWN_PCG_FP32 if main_prec == fs.FS_PRECISION_FP32_REFINE else BYTES_PER_UNKNOWN_PCG_FP64
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
        adjoint = adjoint_steps(fs, n, min(args.warmup, 1), min(args.steps, 2))
        adjoint["ms_per_step"] = max_over_ranks(adjoint["ms_per_step"])

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        iters = fp64["pcg_iterations_per_step"] / 3.0 if fp64 else 400.0
        ref_ms, sample, threads = reference_sample_best(n, iters)
        if ref_ms is not None:
            cpu = {"value": ref_ms, "unit": "ms", "cores": threads, "kind": "reference", "sample": sample}

    line = {
        "metric": metric, "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if main_prec == fs.FS_PRECISION_FP32_REFINE else "f64",
        "data": "synthetic", "config": config,
        "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": "the first %d timed steps replayed from their saved states" % min(args.e2e_steps, args.steps),
                "device_ms_same_steps": e2e_device_ms},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "pressure PCG iteration (spmv + update + direction, 3 kernels)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_src,
                     "traffic": (TRAFFIC_PER_ITERATION_256_FP32 * N / 256 ** 3
                                 if main_prec == fs.FS_PRECISION_FP32_REFINE else None),
                     "traffic_unit": "bytes per PCG iteration (ncu capture at 256^3, scaled by unknowns)",
                     "bytes_per_iteration": bpu * N,
                     "pcg_ms": pcg_ms, "pcg_launched_iterations": pcg_its, "pcg_iterations": real_its},
        "fp64": fp64,
        "adjoint": adjoint,
        "steps_detail": [{k: r[k] for k in ("ms", "pcg_iterations", "outer_iterations", "viscosity_iterations",
                                             "max_rel_residual", "div_linf", "pcg_ms")} for r in reps],
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
