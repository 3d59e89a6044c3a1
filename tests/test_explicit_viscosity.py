"""The reference's air/water viscosity on the GPU (fs_params.viscosity = 2):
the explicit variable-viscosity update of VISCOSITY_3D::ApplyViscosity
(VISCOSITY_3D.h:452-563), through the C ABI.

- in place (FS_FLAG_VISCOSITY_IN_PLACE): x, then y, then z, each in (k, j, i)
  order as the reference's single thread runs it, against the goldens the
  compiled reference produced (FP64, to rounding: the Heaviside's sine is the
  only operation that may differ in the last bit);
- corrected: one explicit Euler step from the input velocities, against the
  oracle in FP64 and FP32;
- the explicit viscous term of the CFL condition (EULERIAN_FLUID_SOLVER_3D.h:2765-2768);
- whole timesteps with the explicit viscosity against the oracle's step."""
import os

import numpy as np
import pytest

import fluid_simulator_backup_b200 as fs
from oracle import fs_oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def solver(g, precision=fs.FS_PRECISION_FP64, flags=0, **kw):
    n = int(g["n"])
    return fs.Solver(n, float(g["dx"]), precision=precision, rho_neg=float(g["rho_neg"]),
                     rho_pos=float(g["rho_pos"]), mu_neg=float(g["mu_neg"]), mu_pos=float(g["mu_pos"]), viscosity=2,
                     flags=flags, **kw)


@pytest.mark.parametrize("name", ["explicit_viscosity_drop", "explicit_viscosity_bubble"])
def test_in_place_explicit_viscosity_matches_reference_golden(name):
    g = load(name)
    with solver(g, flags=fs.FS_FLAG_VISCOSITY_IN_PLACE) as s:
        for k in ("phi", "u", "v", "w"):
            s.upload(k, g[k])
        assert s.viscosity(float(g["dt"])) == 0
        for k in "uvw":
            out = s.download(k)
            step = np.abs(g["out_" + k] - g[k]).max()
            assert np.abs(out - g["out_" + k]).max() <= 1e-10 * step + 1e-15, k


@pytest.mark.parametrize("precision,tol", [(fs.FS_PRECISION_FP64, 1e-10), (fs.FS_PRECISION_FP32_REFINE, 1e-4)])
def test_corrected_explicit_viscosity_matches_oracle(precision, tol):
    g = load("explicit_viscosity_bubble")
    args = (g["phi"], g["u"], g["v"], g["w"], float(g["dx"]), float(g["dt"]), float(g["rho_neg"]),
            float(g["rho_pos"]), float(g["mu_neg"]), float(g["mu_pos"]))
    ref = O.explicit_viscosity(*args, faithful=False)
    with solver(g, precision=precision) as s:
        for k in ("phi", "u", "v", "w"):
            s.upload(k, g[k])
        s.viscosity(float(g["dt"]))
        for k, r, x0 in zip("uvw", ref, (g["u"], g["v"], g["w"])):
            out = s.download(k)
            step = np.abs(r - x0).max()
            # the increment is compared relative to its own size (FP32: the
            # stored velocity rounds at eps32 |u| as well)
            floor = 0.0 if precision == fs.FS_PRECISION_FP64 else 2e-7 * np.abs(x0).max()
            assert np.abs(out - r).max() <= tol * step + floor, k


def test_cfl_includes_the_explicit_viscous_term():
    g = load("explicit_viscosity_bubble")
    n = int(g["n"])
    with solver(g, cfl=1.0) as s:
        for k in ("phi", "u", "v", "w"):
            s.upload(k, g[k])
        dt = s.cfl_dt()
    nu = max(float(g["mu_neg"]) / float(g["rho_neg"]), float(g["mu_pos"]) / float(g["rho_pos"]))
    ref = O.cfl_dt(g["u"], g["v"], g["w"], float(g["dx"]), -9.8, nu_max=nu)
    assert abs(dt - ref) <= 1e-12 * ref
    with fs.Solver(n, float(g["dx"]), viscosity=1, cfl=1.0) as s:  # semi-implicit: no viscous limit
        for k in ("u", "v", "w"):
            s.upload(k, g[k])
        assert abs(s.cfl_dt() - O.cfl_dt(g["u"], g["v"], g["w"], float(g["dx"]), -9.8)) <= 1e-12


@pytest.mark.parametrize("in_place", [False, True])
def test_whole_step_with_explicit_viscosity_matches_oracle(in_place):
    n = 14
    dx = 1.0 / n
    x = (np.arange(n) + 0.5) / n
    phi = np.sqrt((x[None, None, :] - 0.5) ** 2 + (x[None, :, None] - 0.4) ** 2 + (x[:, None, None] - 0.5) ** 2) - 0.25
    rng = np.random.default_rng(8)
    u, v, w = O.zero_walls(rng.normal(size=(n, n, n + 1)) * 0.1, rng.normal(size=(n, n + 1, n)) * 0.1,
                           rng.normal(size=(n + 1, n, n)) * 0.1)
    P = dict(rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, gravity=(0.0, -9.8, 0.0), eps=1e-6,
             reinit_iterations=10, reinit_scaling=5, tol=1e-12, max_iter=20000, viscosity="explicit",
             viscosity_in_place=in_place, visc_tol=1e-12)
    flags = fs.FS_FLAG_VISCOSITY_IN_PLACE if in_place else 0
    with fs.Solver(n, dx, rho_neg=1.0, rho_pos=1000.0, mu_neg=1.8e-5, mu_pos=1e-3, viscosity=2, flags=flags,
                   tolerance=1e-12) as s:
        for k, a in zip(("phi", "u", "v", "w"), (phi, u, v, w)):
            s.upload(k, a)
        dt = s.cfl_dt()
        s.step(dt)
        got = [s.download(k) for k in ("phi", "u", "v", "w")]
    ref = O.step(phi, u, v, w, dx, dt, P)[:4]
    assert rel_err(got[0], ref[0]) < 1e-9
    for a, b in zip(got[1:], ref[1:]):
        assert np.abs(a - b).max() < 1e-8 * max(np.abs(b).max(), 1e-3)
