"""Oil/water vertical pipe mode: the oracle against the reference's own
outputs (fixtures pipe_* made by tests/golden/make_golden.py from the
headless reference build, one reference thread).

The pipe is the reference's production scenario (all four of its .sim files
select it): a periodic vertical pipe of radius a in a box, the core-annular
level set, dimensionless constants derived from the script.  Each operator
here must agree bit for bit."""
import os

import numpy as np

from oracle import fs_oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def grids(g):
    return O.pipe_grids(tuple(int(x) for x in g["n"]), tuple(g["lo"]), tuple(g["hi"]))


def test_pipe_constants_and_boundary_match_reference():
    g = load("pipe_levelset")
    C = O.pipe_constants(float(g["a"]), 0.47625, float(g["m"]), float(g["eta"]), float(g["K"]), float(g["g"]),
                         0.995, float(g["oil_density"]), 0.01, 6.01, 8.54)
    for k in ("R1", "f", "A", "V0", "J", "Re", "We"):
        assert C[k] == float(g[k]), k
    b = O.pipe_boundary(grids(g)[0], g["phi"].shape, float(g["a"]))
    np.testing.assert_array_equal(b, g["boundary"])
    # the pipe keeps at least three cells of the box around it (its WENO5
    # cells never read the box's ghost layers)
    inside = np.argwhere(b <= 0)
    n = g["phi"].shape
    assert inside[:, 0].min() >= 3 and inside[:, 0].max() <= n[0] - 4
    assert inside[:, 2].min() >= 3 and inside[:, 2].max() <= n[2] - 4


def test_pipe_levelset_advection_matches_reference():
    g = load("pipe_levelset")
    phi, u, v, w = O.pipe_weno5_levelset(g["phi"], g["u"], g["v"], g["w"], grids(g), float(g["a"]), float(g["dt"]),
                                         float(g["epsilon"]))
    np.testing.assert_array_equal(phi, g["out_phi"])
    for k, a in zip("uvw", (u, v, w)):
        np.testing.assert_array_equal(a, g["out_" + k])
    # cells outside the pipe keep their value; u and w are zero outside it
    b = g["boundary"]
    np.testing.assert_array_equal(phi[b > 0], g["phi"][b > 0])
    assert (np.abs(phi - g["phi"])[b <= 0] > 0).any()


def test_pipe_reinitialization_matches_reference():
    g = load("pipe_reinit")
    out = O.pipe_reinitialization(g["phi"], grids(g), int(g["reinit_iterations"]), int(g["reinit_scaling"]),
                                  float(g["epsilon"]), typo=True)
    np.testing.assert_array_equal(out, g["out_phi"])


def test_pipe_forcing_matches_reference():
    g = load("pipe_forcing")
    C = {k: float(g[k]) for k in ("a", "R1", "eta", "f", "V0")}
    out = O.pipe_forcing(g["phi"], g["v"], grids(g), C, float(g["gravity_y"]), float(g["oil_density"]),
                         float(g["dt"]), fixed_v=g["fixed_v"])
    np.testing.assert_array_equal(out, g["out_v"])
    np.testing.assert_array_equal(g["out_u"], g["u"])
    np.testing.assert_array_equal(g["out_w"], g["w"])
    # the centre-line faces are fixed and keep their value
    assert g["fixed_v"].sum() > 0
    np.testing.assert_array_equal(out[g["fixed_v"]], g["v"][g["fixed_v"]])


def test_pipe_velocity_advection_matches_reference():
    g = load("pipe_velocity")
    out = O.pipe_eno3_velocity(g["u"], g["v"], g["w"], grids(g), float(g["a"]), float(g["dt"]))
    for k, a in zip("uvw", out):
        np.testing.assert_array_equal(a, g["out_" + k])
    fixed = O.pipe_fixed_faces(tuple(int(x) for x in g["n"]))
    for k, f in zip("uvw", fixed):
        np.testing.assert_array_equal(f, g["fixed_" + k])
        # fixed faces and faces outside the pipe keep their value
        np.testing.assert_array_equal(g["out_" + k][f], g[k][f])


def test_pipe_projection_matches_reference():
    """EULERIAN_FLUID_SOLVER_3D::Projection of the pipe, bit for bit: the
    divergence of the pipe's velocity copies, the deflated system's diagonal,
    right-hand side (jump terms kappa/We, mean removed over the unknowns) and
    solution in the reference's row order, the PCG iteration count, the
    pressure and the updated velocities."""
    g = load("pipe_projection")
    C = {k: float(g[k]) for k in ("a", "R1", "m", "eta", "K", "g", "f", "A", "V0", "J", "Re", "We")}
    fixed = (g["fixed_u"], g["fixed_v"], g["fixed_w"])
    u, v, w, p, info = O.pipe_projection(g["phi"], g["u"], g["v"], g["w"], grids(g), C, float(g["dt"]),
                                         float(g["tolerance"]), int(g["max_iteration"]), float(g["water_density"]),
                                         float(g["oil_density"]), fixed=fixed)
    fl = info["fluid"]
    assert fl.sum() == len(g["b_rows"])
    np.testing.assert_array_equal(info["div"], g["div"])
    np.testing.assert_array_equal(info["jc"][fl], g["jc"][fl])
    vals, rp = g["csr_vals"], g["csr_rowptr"]
    np.testing.assert_array_equal(info["op"][3][fl], vals[rp[1:] - 1])  # the diagonal is each row's last entry
    np.testing.assert_array_equal(info["b"][fl], g["b_rows"])
    assert info["iterations"] == int(g["iterations"])
    np.testing.assert_array_equal(p[fl], g["x_rows"])
    np.testing.assert_array_equal(p, g["out_p"])
    for k, a in zip("uvw", (u, v, w)):
        np.testing.assert_array_equal(a, g["out_" + k])


def test_pipe_cfl_matches_reference():
    """CFLOneTimeStep of the pipe (dimensionless form, semi-implicit
    viscosity) on the projected velocities, with the projection's curvature
    maximum."""
    g = load("pipe_projection")
    C = {k: float(g[k]) for k in ("a", "R1", "m", "eta", "K", "g", "f", "A", "V0", "J", "Re", "We")}
    gr = grids(g)
    _, kmax = O.curvature(g["phi"], gr[0][3], typo=True)
    dt = O.pipe_cfl_dt(g["out_u"], g["out_v"], g["out_w"], gr, C, float(g["gravity_y"]), float(g["water_density"]),
                       float(g["oil_density"]), kmax)
    assert dt == float(g["cfl"])


def test_pipe_frame_matches_reference():
    """One whole SIMULATION_WORLD::AdvanceOneFrame of the pipe with the
    reference's sourcing step off (no viscosity), bit for bit: the CFL dt
    from the level set's curvature, then the order-2 step (level-set Heun,
    velocity Heun over ENO3 advection + body force + projection,
    reinitialisation Heun)."""
    g = load("pipe_frame")
    gr = grids(g)
    C = {k: float(g[k]) for k in ("a", "R1", "m", "eta", "K", "g", "f", "A", "V0", "J", "Re", "We")}
    _, kmax = O.curvature(g["phi"], gr[0][3], typo=True)
    dt = O.pipe_cfl_dt(g["u"], g["v"], g["w"], gr, C, float(g["gravity_y"]), float(g["water_density"]),
                       float(g["oil_density"]), kmax) * float(g["cfl_number"])
    assert dt == float(g["dt"])
    P = dict(tolerance=float(g["tolerance"]), max_iteration=int(g["max_iteration"]),
             water_density=float(g["water_density"]), oil_density=float(g["oil_density"]),
             gravity_y=float(g["gravity_y"]), epsilon=float(g["epsilon"]),
             reinit_iterations=int(g["reinit_iterations"]), reinit_scaling=int(g["reinit_scaling"]))
    out = O.pipe_step(g["phi"], g["u"], g["v"], g["w"], gr, C, dt, P)
    for name, a in zip(("phi", "u", "v", "w", "p"), out):
        np.testing.assert_array_equal(a, g["out_" + name])


def test_pipe_viscosity_matches_reference():
    """VISCOSITY_3D::ApplyViscosity of the pipe (the reference's oil/water
    semi-implicit branch), bit for bit: per component the six coefficients
    and the explicit term on the unknowns (faces inside the pipe), and the
    solved velocities everywhere."""
    g = load("pipe_viscosity")
    gr = grids(g)
    C = {k: float(g[k]) for k in ("a", "R1", "m", "eta", "K", "g", "f", "A", "V0", "J", "Re", "We")}
    u, v, w, info = O.pipe_viscosity(g["phi"], g["u"], g["v"], g["w"], gr, C, float(g["dt"]), float(g["tolerance"]),
                                     int(g["max_iteration"]))
    for a, k in enumerate("uvw"):
        b = O.pipe_boundary(gr[1 + a], g[k].shape, C["a"])
        ny = b.shape[1]
        rows = (b <= 0) & (np.arange(ny)[None, :, None] < (ny - 1 if a == 1 else ny))
        np.testing.assert_array_equal(info["explicit_" + k][rows], g[f"{k}_q0"][rows])
        for q in range(6):
            np.testing.assert_array_equal(info["coef_" + k][q][rows], g[f"{k}_q{q + 1}"][rows])
    for k, a in zip("uvw", (u, v, w)):
        np.testing.assert_array_equal(a, g["out_" + k])


def test_pipe_frame_with_viscosity_matches_reference():
    """One whole AdvanceOneFrame of the pipe as the reference's own pipe
    scripts run it (sourcing on: the semi-implicit viscosity between the
    body force and the projection in each velocity stage, the fixed
    centre-line faces kept), bit for bit, dt included."""
    g = load("pipe_frame_viscous")
    gr = grids(g)
    C = {k: float(g[k]) for k in ("a", "R1", "m", "eta", "K", "g", "f", "A", "V0", "J", "Re", "We")}
    _, kmax = O.curvature(g["phi"], gr[0][3], typo=True)
    dt = O.pipe_cfl_dt(g["u"], g["v"], g["w"], gr, C, float(g["gravity_y"]), float(g["water_density"]),
                       float(g["oil_density"]), kmax) * float(g["cfl_number"])
    assert dt == float(g["dt"])
    P = dict(tolerance=float(g["tolerance"]), max_iteration=int(g["max_iteration"]),
             water_density=float(g["water_density"]), oil_density=float(g["oil_density"]),
             gravity_y=float(g["gravity_y"]), epsilon=float(g["epsilon"]),
             reinit_iterations=int(g["reinit_iterations"]), reinit_scaling=int(g["reinit_scaling"]), sourcing=True)
    out = O.pipe_step(g["phi"], g["u"], g["v"], g["w"], gr, C, dt, P)
    for name, a in zip(("phi", "u", "v", "w", "p"), out):
        np.testing.assert_array_equal(a, g["out_" + name])
