"""The adjoint at 512^3 (134 M cells): the oil/water Rayleigh-Taylor scene in
the FP32 + FP64 refinement path with semi-implicit viscosity, a short
forward lead-in, then the gradient of L = ||phi(T)||^2 over a window of 16
steps through the torch.autograd rollout with Griewank's binomial
checkpointing (3 snapshots), reporting the peak device memory of the
context (fields, tape, adjoint buffers) and of the device.  The adjoint's
derivatives themselves are checked against finite differences at small
sizes (test_adjoint.py, test_adjoint_fp32.py); here the 512^3 window must
run within one B200's memory and give finite bars."""
import numpy as np
import pytest

import fluid_simulator_backup_b200 as fs

pytestmark = pytest.mark.gpu

LEAD_IN = 2
WINDOW = 16


def rayleigh_taylor(n, seed=0):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(8, 8))
    px, pz = rng.uniform(0, 1, size=(8, 8)), rng.uniform(0, 1, size=(8, 8))
    xs = (np.arange(n) + 0.5) / n
    pert = np.zeros((n, n))  # [z, x]
    for kx in range(8):
        for kz in range(8):
            pert += a[kx, kz] * np.cos(2 * np.pi * ((kx + 1) * xs[None, :] + px[kx, kz])) * \
                np.cos(2 * np.pi * ((kz + 1) * xs[:, None] + pz[kx, kz]))
    pert *= 0.01 / np.abs(pert).max()
    return (xs[None, :, None] - 0.5) - pert[:, None, :]


def test_rayleigh_taylor_512_adjoint_window():
    import torch

    from rollout import Rollout, Schedule
    n = 512
    dx = 1.0 / n
    free0, total = torch.cuda.mem_get_info()
    with fs.Solver(n, dx, rho_neg=850.0, rho_pos=1000.0, mu_neg=5e-2, mu_pos=1e-3,
                   precision=fs.FS_PRECISION_FP32_REFINE, tolerance=1e-6, stop=fs.FS_STOP_RELATIVE,
                   max_iteration=20000, cfl=0.5, order=3, viscosity=1, viscosity_tolerance=1e-8) as s:
        s.upload("phi", rayleigh_taylor(n))
        for k in ("u", "v", "w"):
            s.upload(k, np.zeros(s.shape(k)))
        dt = s.cfl_dt()
        for _ in range(LEAD_IN):
            s.step(dt)
        X = {k: s.download(k) for k in ("phi", "u", "v", "w")}
        ts = {k: torch.tensor(X[k], requires_grad=True) for k in X}
        rho = torch.tensor(850.0, dtype=torch.float64, requires_grad=True)
        sched = Schedule()
        out = Rollout.apply(ts["phi"], ts["u"], ts["v"], ts["w"], rho, s, dt, WINDOW, 3, sched, "neg")
        loss = torch.sum(out[0] ** 2)
        loss.backward()
        lib_bytes = s.memory_bytes()
        free1, _ = torch.cuda.mem_get_info()
        grads = {k: ts[k].grad.numpy() for k in X}
    peak_dev = total - free1
    print(f"512^3 adjoint of {WINDOW} steps (binomial, 3 snapshots): {sched.forward_steps} forward steps, "
          f"{sched.adjoint_steps} adjoint steps, context {lib_bytes / 2**30:.1f} GiB, device in use "
          f"{peak_dev / 2**30:.1f} GiB of {total / 2**30:.1f} GiB, d loss / d rho_oil = {float(rho.grad):.6e}")
    assert sched.adjoint_steps == WINDOW and sched.max_live_snapshots <= 3
    assert all(np.isfinite(g).all() for g in grads.values())
    assert np.isfinite(float(rho.grad))
    assert lib_bytes < 170 * 2**30
