"""Generate the golden vectors in tests/golden/ from the reference's own code.

Runs the reference solver built headlessly (oracle/refbuild -> oracle/_ref/
libfsref.so) on seeded synthetic inputs and stores inputs and outputs as
.npz fixtures.  The fixtures travel with the repository; the reference build
does not have to exist where the tests run.

    python tests/golden/make_golden.py      (from the repository root)

Every case is a single reference operator called with number_of_threads = 1
on the air/water unit-cube box with Neumann pressure walls:
  weno5_levelset   ADVECTION_METHOD_3D<T>::WENO5th on the level set
  weno5_velocity   WENO5th on u, v, w (each with its own ghost copy)
  reinit           one Reinitialization block (sign function + 10 Sussman
                   pseudo-steps), ghosts re-extrapolated before each step
  projection_*     PROJECTION_3D::Solve: divergence, CSR system, PCG, velocity
                   update (the reference as it runs: only w corrected)
  semi_implicit_*  POISSON_SOLVER_3D::SolveForViscosity on seeded coefficients
  cfl              EULERIAN_FLUID_SOLVER_3D::CFLOneTimeStep
  projection_tension  curvature (LEVELSET_3D::ComputeCurvatures) and
                   PROJECTION_3D::Solve with a surface tension jump condition
  levelset_file    the bytes LEVELSET_3D::Write produces for a level set
  eno3_velocity    ADVECTION_METHOD_3D<T>::ENO3rd on u, v, w
  fast_sweeping    LEVELSET_3D::FastSweepingMethod (after its ghost fill) on a
                   noisy sphere, sweep_direction 0 and 3; inputs whose sort
                   never reads the uninitialised a2 of INCREASING_SORT3's
                   typo branch (checked with the oracle)
  surface_*        MARCHING_CUBES_ALGORITHM::Polygonize as WRITE_LEVELSET::
                   WriteOBJ runs it (after ComputeNormals): vertices, vertex
                   normals, triangles (1-based) of a sphere (16^3) and a
                   noisy scaled sphere (24^3)
  explicit_viscosity_*  VISCOSITY_3D::ApplyViscosity, the air/water explicit
                   in-place update (x, then y, then z), on a noisy sphere with
                   random velocities, both phase conventions (10^3); the level
                   set's first ghost layer is the oracle's linear
                   extrapolation and the velocity ghosts are zero
  pipe_levelset    oil/water vertical pipe: ADVECTION_3D::Solve_Levelset (the
                   cylinder's velocity set-up, periodic ghosts, WENO5 skipping
                   cells outside the pipe)
  pipe_velocity    the pipe's ADVECTION_3D::Solve_Velocity with ENO3: masked
                   periodic ghost copies with the wall extrapolation, the
                   guarded copies of the ENO stencils, fixed centre-line faces
  pipe_reinit      the pipe's Reinitialization (sign function + 10 Sussman
                   pseudo-steps on periodic ghosts)
  pipe_forcing     the pipe's dimensionless body force (ApplyGravity), with
                   the centre-line faces that Solve_Velocity marks fixed
  pipe_projection  the pipe's Projection: Neumann cells outside the
                   cylinder, the pipe divergence, jump 1/We kappa, the
                   deflated system (right-hand side and solution in row
                   order), PCG and the pipe velocity update; then the
                   pipe's CFLOneTimeStep
  pipe_viscosity   the pipe's VISCOSITY_3D::ApplyViscosity (oil/water
                   semi-implicit branch): per component the explicit term,
                   coef_1..coef_6 and the solved velocity
  pipe_frame       one SIMULATION_WORLD::AdvanceOneFrame of the pipe with
                   is_sourcing_active = false (no viscosity): CFL dt and the
                   order-2 step
  pipe_frame_viscous  the same frame with sourcing on, as the reference's own
                   pipe scripts run it (semi-implicit viscosity in each stage)

    python tests/golden/make_golden.py [name ...]   writes only the named fixtures
"""
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)
from oracle import fs_oracle  # noqa: E402
from oracle import refsim  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
WORK = os.path.join(OUT, "_sim")


def sphere(n, c, r):
    x = (np.arange(n) + 0.5) / n
    return np.sqrt((x[None, None, :] - c[0]) ** 2 + (x[None, :, None] - c[1]) ** 2 + (x[:, None, None] - c[2]) ** 2) - r


def box_sdf(n, hi):
    """Signed distance to the box [0,hi0]x[0,hi1]x[0,hi2] at cell centres
    (negative inside); the dam-break initial level set."""
    x = (np.arange(n) + 0.5) / n
    X, Y, Z = x[None, None, :], x[None, :, None], x[:, None, None]
    q = [np.abs(X - hi[0] / 2) - hi[0] / 2, np.abs(Y - hi[1] / 2) - hi[1] / 2, np.abs(Z - hi[2] / 2) - hi[2] / 2]
    outside = np.sqrt(sum(np.maximum(a, 0.0) ** 2 for a in q))
    inside = np.minimum(np.maximum(np.maximum(q[0], q[1]), q[2]), 0.0)
    return outside + inside


def case(n, **kw):
    os.makedirs(WORK, exist_ok=True)
    path = refsim.write_sim(os.path.join(WORK, f"case_{n}.sim"), n, **kw)
    return refsim.RefCase(path)


def main():
    rng = np.random.default_rng(20241203)
    fixtures = {}

    # WENO5 level set, random field and random face velocities, 11^3
    n = 11
    c = case(n)
    phi = rng.normal(size=c.shape("phi")) * 0.1
    vel = {k: rng.normal(size=c.shape(k)) * 0.3 for k in "uvw"}
    for k, a in vel.items():
        c.set(k, a)
    c.set("phi", phi)
    c.weno5_levelset(2e-3)
    fixtures["weno5_levelset"] = dict(n=n, dx=c.dx, dt=2e-3, eps=1e-6, phi=phi, **vel, out=c.get("phi"))
    c.close()

    # WENO5 MAC self-advection, 10^3
    n = 10
    c = case(n)
    vel = {k: rng.normal(size=c.shape(k)) * 0.3 for k in "uvw"}
    for k, a in vel.items():
        c.set(k, a)
    c.weno5_velocity(2e-3, 1)
    fixtures["weno5_velocity"] = dict(n=n, dx=c.dx, dt=2e-3, eps=1e-6, **vel,
                                      out_u=c.get("u"), out_v=c.get("v"), out_w=c.get("w"))
    c.close()

    # Sussman reinitialisation block on a noisy field (exercises every branch
    # of the Godunov case tree), 12^3
    n = 12
    c = case(n)
    phi = rng.normal(size=c.shape("phi")) * 0.1
    c.set("phi", phi)
    c.reinitialization(1e-3, 1)
    fixtures["reinit"] = dict(n=n, dx=c.dx, iterations=10, scaling=5, eps=1e-6, phi=phi, out=c.get("phi"))
    c.close()

    # Projection, both phase conventions, 10^3.  The reference's curvature
    # routine (called inside the projection for the jump term) exits the
    # process where the central-difference gradient vanishes
    # (LEVELSET_3D.h:1040-1044); the box SDF has such points on its medial
    # planes, so it gets a small seeded perturbation.
    n = 10
    drop_phi = box_sdf(n, (0.4, 0.6, 1.0)) + 1e-3 * rng.normal(size=(n, n, n))
    for name, water_drop, phi in (("projection_drop", True, drop_phi),
                                  ("projection_bubble", False, sphere(n, (0.5, 0.4, 0.5), 0.3))):
        c = case(n, water_drop=water_drop, tolerance=1e-9)
        vel = {k: rng.normal(size=c.shape(k)) * 0.3 for k in "uvw"}
        for k, a in vel.items():
            c.set(k, a)
        c.set("phi", phi)
        it = c.projection(2e-3)
        vals, cols, rowptr, b, x = c.poisson_csr()
        fixtures[name] = dict(n=n, dx=c.dx, dt=2e-3, tol=1e-9, rho_neg=1000.0 if water_drop else 1.0,
                              rho_pos=1.0 if water_drop else 1000.0, phi=phi, **vel, iterations=it,
                              csr_vals=vals, csr_cols=cols, csr_rowptr=rowptr, b=b, x=x,
                              div=c.divergence(), out_p=c.get("p"), out_u=c.get("u"), out_v=c.get("v"),
                              out_w=c.get("w"))
        c.close()

    # Semi-implicit viscosity systems, 8^3
    n = 8
    c = case(n, tolerance=1e-9)
    for axis, k in enumerate("uvw"):
        shp = c.shape(k)
        coef = rng.uniform(0.01, 0.3, size=(6,) + shp) * c.dx * c.dx
        ex = rng.normal(size=shp)
        comp0 = rng.normal(size=shp) * 0.1
        c.set(k, comp0)
        out, it = c.semi_implicit_solve(axis + 1, coef, ex)
        fixtures[f"semi_implicit_{k}"] = dict(n=n, dx=c.dx, tol=1e-9, axis=axis, coef=coef, explicit=ex,
                                             comp0=comp0, out=out, iterations=it)
    c.close()

    # CFL dt, 9^3
    n = 9
    c = case(n)
    vel = {k: rng.normal(size=c.shape(k)) * s for k, s in zip("uvw", (0.5, 1.5, 0.7))}
    for k, a in vel.items():
        c.set(k, a)
    fixtures["cfl"] = dict(n=n, dx=c.dx, gravity_y=-9.8, nu_max=max(1e-3 / 1000.0, 1.8e-5 / 1.0), **vel, out=c.cfl())
    c.close()

    # Surface tension (sigma = 0.0728, air bubble in water), 10^3: the
    # curvature of a perturbed sphere (LEVELSET_3D::ComputeCurvatures) and a
    # projection whose right-hand side and velocity update carry the jump
    # condition sigma*kappa
    n = 10
    c = case(n, water_drop=False, tolerance=1e-9, surface_tension=0.0728)
    phi = sphere(n, (0.5, 0.4, 0.5), 0.3) + 1e-3 * rng.normal(size=(n, n, n))
    vel = {k: rng.normal(size=c.shape(k)) * 0.3 for k in "uvw"}
    for k, a in vel.items():
        c.set(k, a)
    c.set("phi", phi)
    kappa = c.curvature()
    it = c.projection(2e-3)
    vals, cols, rowptr, b, x = c.poisson_csr()
    fixtures["projection_tension"] = dict(n=n, dx=c.dx, dt=2e-3, tol=1e-9, rho_neg=1.0, rho_pos=1000.0, sigma=0.0728,
                                          phi=phi, **vel, kappa=kappa, iterations=it, csr_vals=vals, csr_cols=cols,
                                          csr_rowptr=rowptr, b=b, x=x, out_p=c.get("p"), out_u=c.get("u"),
                                          out_v=c.get("v"), out_w=c.get("w"))
    c.close()

    # A level set written by LEVELSET_3D::Write (the bytes of the file), 9^3
    n = 9
    c = case(n)
    phi = rng.normal(size=c.shape("phi"))
    c.set("phi", phi)
    path = os.path.join(WORK, "levelset.bin")
    c.write_levelset(path)
    with open(path, "rb") as f:
        raw = np.frombuffer(f.read(), dtype=np.uint8).copy()
    fixtures["levelset_file"] = dict(n=n, dx=c.dx, phi=phi, raw=raw)
    c.close()

    # ENO3 MAC self-advection (the scheme the reference's own scripts select
    # for velocity, use_3rd_eno_v), 10^3
    n = 10
    c = case(n, velocity_weno=False)
    vel = {k: rng.normal(size=c.shape(k)) * 0.3 for k in "uvw"}
    for k, a in vel.items():
        c.set(k, a)
    c.eno3_velocity(2e-3)
    fixtures["eno3_velocity"] = dict(n=n, dx=c.dx, dt=2e-3, **vel, out_u=c.get("u"), out_v=c.get("v"),
                                     out_w=c.get("w"))
    c.close()

    # fast sweeping reinitialisation, 20^3: a sphere scaled by 1.5 plus noise
    n = 20
    c = case(n, water_drop=False)
    frng = np.random.default_rng(3)
    phi = sphere(n, (0.5, 0.45, 0.5), 0.3) * 1.5 + frng.normal(size=(n, n, n)) * 0.01
    outs = {}
    for direction in (0, 3):
        c.set("phi", phi)
        c.fast_sweeping(direction)
        outs[f"out_{direction}"] = c.get("phi")
    fixtures["fast_sweeping"] = dict(n=n, dx=c.dx, phi=phi, **outs)
    c.close()

    # the level set's surface as the OBJ writer makes it
    for name, n, scale, noise in (("surface_sphere", 16, 1.0, 0.0), ("surface_noisy", 24, 1.3, 0.002)):
        c = case(n, water_drop=False)
        srng = np.random.default_rng(1)
        phi = sphere(n, (0.5, 0.45, 0.5), 0.3) * scale + srng.normal(size=(n, n, n)) * noise
        c.set("phi", phi)
        xyz, nrm, tri = c.marching_cubes()
        fixtures[name] = dict(n=n, dx=c.dx, phi=phi, xyz=xyz, normals=nrm, tri=tri)
        c.close()

    # explicit air/water viscosity (its own seed: the fixtures above keep their draws)
    vrng = np.random.default_rng(11)
    n = 10
    for name, water_drop in (("explicit_viscosity_drop", True), ("explicit_viscosity_bubble", False)):
        c = case(n, water_drop=water_drop)
        phi = sphere(n, (0.5, 0.45, 0.5), 0.3) + vrng.normal(size=(n, n, n)) * 0.02
        vel = {k: vrng.normal(size=c.shape(k)) * 0.3 for k in "uvw"}
        for k, a in vel.items():
            c.set(k, a)
        c.set("phi", phi)
        c.viscosity_ghosted(fs_oracle.extrapolate_ghosts(phi, 1), 2e-3)
        fixtures[name] = dict(n=n, dx=c.dx, dt=2e-3, rho_neg=1000.0 if water_drop else 1.0,
                              rho_pos=1.0 if water_drop else 1000.0, mu_neg=1e-3 if water_drop else 1.8e-5,
                              mu_pos=1.8e-5 if water_drop else 1e-3, phi=phi, **vel, out_u=c.get("u"),
                              out_v=c.get("v"), out_w=c.get("w"))
        c.close()

    # oil/water vertical pipe (the reference's production mode): a 21 x 16 x
    # 21 cell grid of spacing 0.25 around a pipe of radius a = 1.61, the
    # constants of its 3D_script_1.sim; level set = the reference's own
    # core-annular seed plus noise, face velocities random around the
    # dimensionless core flow
    h, pn = 0.25, (21, 16, 21)
    lo = (-(pn[0] - 1) / 2 * h, 0.0, -(pn[2] - 1) / 2 * h)
    hi = ((pn[0] - 1) / 2 * h, (pn[1] - 1) * h, (pn[2] - 1) / 2 * h)
    pipe_sim = refsim.write_pipe_sim(os.path.join(WORK, "pipe.sim"), pn, lo, hi)
    rng = np.random.default_rng(11)
    c = refsim.RefCase(pipe_sim)
    const = c.pipe_params()
    phi = c.get("phi") + rng.normal(0.0, 0.02, c.shape("phi"))
    vel = dict(u=rng.normal(0.0, 0.3, c.shape("u")), v=1.0 + rng.normal(0.0, 0.3, c.shape("v")),
               w=rng.normal(0.0, 0.3, c.shape("w")))
    base = dict(n=pn, lo=lo, hi=hi, boundary=c.boundary_levelset(),
                **{k: const[k] for k in ("a", "R1", "m", "eta", "K", "g", "f", "A", "V0", "J", "Re", "We")},
                oil_density=const["oil_density"], gravity_y=-980.0, reinit_iterations=10, reinit_scaling=2,
                epsilon=1e-6, phi=phi, **vel)
    c.close()
    c = refsim.RefCase(pipe_sim)
    for k, a_ in dict(phi=phi, **vel).items():
        c.set(k, a_)
    c.pipe_levelset_advection(0.01)
    fixtures["pipe_levelset"] = dict(base, dt=0.01, out_phi=c.get("phi"), out_u=c.get("u"), out_v=c.get("v"),
                                     out_w=c.get("w"))
    c.close()
    c = refsim.RefCase(pipe_sim)
    for k, a_ in dict(phi=phi, **vel).items():
        c.set(k, a_)
    c.pipe_velocity_advection(0.01)
    fixtures["pipe_velocity"] = dict(base, dt=0.01, out_u=c.get("u"), out_v=c.get("v"), out_w=c.get("w"),
                                     fixed_u=c.fixed("u"), fixed_v=c.fixed("v"), fixed_w=c.fixed("w"))
    c.close()
    c = refsim.RefCase(pipe_sim)
    c.set("phi", phi)
    c.pipe_reinitialization(0.01)
    fixtures["pipe_reinit"] = dict(base, out_phi=c.get("phi"))
    c.close()
    c = refsim.RefCase(pipe_sim)
    for k, a_ in dict(phi=phi, **vel).items():
        c.set(k, a_)
    c.pipe_velocity_advection(0.0)  # marks the centre-line faces fixed (ADVECTION_3D.h:246-275)
    fixed_v = c.fixed("v")
    for k, a_ in dict(phi=phi, **vel).items():
        c.set(k, a_)
    c.pipe_gravity(0.01)
    fixtures["pipe_forcing"] = dict(base, dt=0.01, fixed_v=fixed_v, out_u=c.get("u"), out_v=c.get("v"),
                                    out_w=c.get("w"))
    c.close()
    # the pipe's projection (EULERIAN_FLUID_SOLVER_3D::Projection): the
    # centre-line faces marked fixed first, as in a run; the previous
    # pressure of a fresh case is 0; the system's right-hand side and
    # solution in the reference's row order pin the matrix assembly
    c = refsim.RefCase(pipe_sim)
    for k, a_ in dict(phi=phi, **vel).items():
        c.set(k, a_)
    c.pipe_velocity_advection(0.0)
    fixed = {f"fixed_{k}": c.fixed(k) for k in "uvw"}
    for k, a_ in dict(phi=phi, **vel).items():
        c.set(k, a_)
    it = c.pipe_projection(0.01)
    cfl = c.cfl()  # CFLOneTimeStep on the projected velocities and the projection's curvature
    vals, cols, rowptr, b_rows, x_rows = c.poisson_csr()
    fixtures["pipe_projection"] = dict(base, dt=0.01, tolerance=1e-6, max_iteration=10000, **fixed,
                                       water_density=const["water_density"], iterations=it, cfl=cfl,
                                       div=c.divergence(), jc=c.projection_jc(), csr_vals=vals, csr_cols=cols,
                                       csr_rowptr=rowptr, b_rows=b_rows, x_rows=x_rows, out_p=c.get("p"),
                                       out_u=c.get("u"), out_v=c.get("v"), out_w=c.get("w"))
    c.close()

    # the pipe's semi-implicit viscosity (VISCOSITY_3D::ApplyViscosity, the
    # oil/water branch): every component's coefficients and explicit term
    # and the solved velocities
    c = refsim.RefCase(pipe_sim)
    for k, a_ in dict(phi=phi, **vel).items():
        c.set(k, a_)
    c.pipe_viscosity(0.01)
    vf = {f"{comp}_q{q}": c.visc_field(comp, q) for comp in "uvw" for q in range(7)}
    fixtures["pipe_viscosity"] = dict(base, dt=0.01, tolerance=1e-6, max_iteration=10000, **vf,
                                      out_u=c.get("u"), out_v=c.get("v"), out_w=c.get("w"))
    c.close()

    # one whole frame of the pipe with the reference's sourcing step off
    # (is_sourcing_active = false: no viscosity), SIMULATION_WORLD::
    # AdvanceOneFrame: curvature, CFL dt, order-2 step (level-set Heun,
    # velocity Heun over ENO3 advection + body force + projection,
    # reinitialisation Heun); the level set and velocities of the other pipe
    # fixtures
    frame_sim = refsim.write_pipe_sim(os.path.join(WORK, "pipe_frame.sim"), pn, lo, hi, sourcing=False)
    c = refsim.RefCase(frame_sim)
    for k, a_ in dict(phi=phi, **vel).items():
        c.set(k, a_)
    dt, it = c.advance_frame()
    fixtures["pipe_frame"] = dict(base, cfl_number=0.8, tolerance=1e-6, max_iteration=10000,
                                  water_density=const["water_density"], dt=dt, iterations=it,
                                  out_phi=c.get("phi"), out_u=c.get("u"), out_v=c.get("v"), out_w=c.get("w"),
                                  out_p=c.get("p"))
    c.close()

    # the same frame as the reference's own pipe scripts run it, sourcing on
    # (the semi-implicit viscosity in every velocity stage)
    c = refsim.RefCase(pipe_sim)
    for k, a_ in dict(phi=phi, **vel).items():
        c.set(k, a_)
    dt, it = c.advance_frame()
    fixtures["pipe_frame_viscous"] = dict(base, cfl_number=0.8, tolerance=1e-6, max_iteration=10000,
                                          water_density=const["water_density"], dt=dt, iterations=it,
                                          out_phi=c.get("phi"), out_u=c.get("u"), out_v=c.get("v"),
                                          out_w=c.get("w"), out_p=c.get("p"))
    c.close()

    only = set(sys.argv[1:])
    for name, d in fixtures.items():
        if only and name not in only:
            continue
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **{k: np.asarray(v) for k, v in d.items()})
        print("wrote", name)
    for f in os.listdir(WORK):
        os.remove(os.path.join(WORK, f))
    os.rmdir(WORK)


if __name__ == "__main__":
    main()
