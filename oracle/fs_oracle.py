"""FP64 CPU restatement of the reference solver's per-timestep hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: `tests/`,
`__graft_entry__.smoke()` and the `cpu_baseline` leg of `bench.py` may call it,
the product path (the CUDA library and its host mirror) never does.

Parity status: pinned.  Each operator below is checked against golden vectors
produced by the reference's own code built headlessly (oracle/refbuild ->
oracle/_ref/libfsref.so, fixtures in tests/golden/).

Layout: cell arrays are [nz, ny, nx] (x fastest, the reference's ARRAY_3D
order, ARRAY_3D.h:98); MAC face arrays carry one extra entry on their own
axis: u [nz, ny, nx+1], v [nz, ny+1, nx], w [nz+1, ny, nx].

Arithmetic follows the reference expression by expression (same operand order
and the same divisions), so with a single thread the stencil operators agree
bit for bit; sums that the reference accumulates sequentially (dot products,
the right-hand-side mean) are accumulated sequentially here too (`_seqsum`).

Two modes exist where the reference's executed air/water step is defective:
`faithful` reproduces the reference operator as it runs; `corrected` is the
specification the GPU path implements.  Differences are listed per function.
"""
import math

import numpy as np

PI = 3.14159265358979323846  # MACROS.h:13
G = 3                        # ghost width of the reference's ghost copies


# ----------------------------------------------------------------------------
# helpers
# ----------------------------------------------------------------------------

def _seqsum(a):
    """Sequential left-to-right sum (the reference's single-thread order)."""
    a = np.ravel(a)
    if a.size == 0:
        return 0.0
    return float(np.cumsum(a)[-1])


def _seqdot(a, b):
    return _seqsum(np.ravel(a) * np.ravel(b))


def face_shape(n, axis):
    nx, ny, nz = n
    return {0: (nz, ny, nx + 1), 1: (nz, ny + 1, nx), 2: (nz + 1, ny, nx)}[axis]


def extrapolate_ghosts(phi, g=G):
    """Ghosted copy of a cell field, linear extrapolation outward.

    Faces follow FillGhostCellsContinuousDerivativesFrom
    (FIELD_STRUCTURE_3D.h:1776-1895): ghost(-m) = 2*ghost(-m+1) - ghost(-m+2)
    evaluated outward, i.e. (1+m)*phi0 - m*phi1.  Edges and corners, which the
    reference fills only partially (three edges, FIELD_STRUCTURE_3D.h:1897-1940,
    the rest commented out), are defined here by extending x first, then y over
    the x-extended rows, then z: the same face values, and a well-defined edge.
    Layout of the result: [nz+2g, ny+2g, nx+2g].
    """
    nz, ny, nx = phi.shape
    a = np.zeros((nz + 2 * g, ny + 2 * g, nx + 2 * g))
    a[g:g + nz, g:g + ny, g:g + nx] = phi
    for m in range(1, g + 1):  # x
        a[g:g + nz, g:g + ny, g - m] = 2.0 * a[g:g + nz, g:g + ny, g - m + 1] - a[g:g + nz, g:g + ny, g - m + 2]
        a[g:g + nz, g:g + ny, g + nx - 1 + m] = 2.0 * a[g:g + nz, g:g + ny, g + nx - 2 + m] - a[g:g + nz, g:g + ny, g + nx - 3 + m]
    for m in range(1, g + 1):  # y
        a[g:g + nz, g - m, :] = 2.0 * a[g:g + nz, g - m + 1, :] - a[g:g + nz, g - m + 2, :]
        a[g:g + nz, g + ny - 1 + m, :] = 2.0 * a[g:g + nz, g + ny - 2 + m, :] - a[g:g + nz, g + ny - 3 + m, :]
    for m in range(1, g + 1):  # z
        a[g - m] = 2.0 * a[g - m + 1] - a[g - m + 2]
        a[g + nz - 1 + m] = 2.0 * a[g + nz - 2 + m] - a[g + nz - 3 + m]
    return a


def zero_ghosts(f, g=G):
    """Ghosted copy with zero ghost values (FillGhostCellsZero,
    FIELD_STRUCTURE_3D.h:538-661, with edges and corners also zero)."""
    return np.pad(f, g)


# ----------------------------------------------------------------------------
# WENO5 (ADVECTION_METHOD_3D.h:42-279)
# ----------------------------------------------------------------------------

def _shift(fg, axis, s, g=G):
    """View of the ghosted array fg shifted by s along `axis` over the
    interior of the un-ghosted field."""
    sl = [slice(g, fg.shape[d] - g) for d in range(3)]
    ax = 2 - axis  # numpy axis of x is 2
    sl[ax] = slice(g + s, fg.shape[ax] - g + s)
    return fg[tuple(sl)]


def _weno_smoothness(a, b, c, first):
    # (T)13/12*(..)*(..) + (T)1/4*(..)*(..), ADVECTION_METHOD_3D.h:97-99
    c1312 = 13.0 / 12.0
    t = (a - 2.0 * b) + c
    if first == 1:
        q = (a - 4.0 * b) + 3.0 * c
    elif first == 2:
        q = a - c
    else:
        q = (3.0 * a - 4.0 * b) + c
    return (c1312 * t) * t + (0.25 * q) * q


def _weno_side(r1, r2, r3, r4, r5, eps):
    s1 = _weno_smoothness(r1, r2, r3, 1)
    s2 = _weno_smoothness(r2, r3, r4, 2)
    s3 = _weno_smoothness(r3, r4, r5, 3)
    a1 = (1.0 / 10.0 * 1.0) / ((eps + s1) * (eps + s1))
    a2 = (6.0 / 10.0 * 1.0) / ((eps + s2) * (eps + s2))
    a3 = (3.0 / 10.0 * 1.0) / ((eps + s3) * (eps + s3))
    sm = (a1 + a2) + a3
    w1, w2, w3 = a1 / sm, a2 / sm, a3 / sm
    t1 = (r1 * 1.0 / 3.0 - r2 * 7.0 / 6.0) + r3 * 11.0 / 6.0
    t2 = (r2 * (-1.0 / 6.0) + r3 * 5.0 / 6.0) + r4 * 1.0 / 3.0
    t3 = (r3 * 1.0 / 3.0 + r4 * 5.0 / 6.0) - r5 * 1.0 / 6.0
    return (w1 * t1 + w2 * t2) + w3 * t3


def weno5_derivatives(fg, axis, inv_h, eps, g=G):
    """One-sided WENO5 derivatives D-, D+ along `axis` of a ghosted field."""
    f = lambda s: _shift(fg, axis, s, g)
    m1 = inv_h * (f(-2) - f(-3))
    m2 = inv_h * (f(-1) - f(-2))
    m3 = inv_h * (f(0) - f(-1))
    m4 = inv_h * (f(1) - f(0))
    m5 = inv_h * (f(2) - f(1))
    p1 = inv_h * (f(3) - f(2))
    p2 = inv_h * (f(2) - f(1))
    p3 = inv_h * (f(1) - f(0))
    p4 = inv_h * (f(0) - f(-1))
    p5 = inv_h * (f(-1) - f(-2))
    return _weno_side(m1, m2, m3, m4, m5, eps), _weno_side(p1, p2, p3, p4, p5, eps)


def _upwind_update(rho, dt, uvel, vvel, wvel, dxm, dxp, dym, dyp, dzm, dzp):
    dx_ = np.where(uvel > 0, dxm, dxp)
    dy_ = np.where(vvel > 0, dym, dyp)
    dz_ = np.where(wvel > 0, dzm, dzp)
    return rho - dt * ((uvel * dx_ + vvel * dy_) + wvel * dz_)


def weno5_levelset(phi, u, v, w, dx, dt, eps):
    """phi - dt*(u.grad phi) with WENO5 upwind derivatives; the upwind side
    is the sign of the cell-averaged face velocity.  The stencil source is the
    linearly extrapolated ghost copy of the current phi."""
    inv = 1.0 / dx
    pg = extrapolate_ghosts(phi)
    dxm, dxp = weno5_derivatives(pg, 0, inv, eps)
    dym, dyp = weno5_derivatives(pg, 1, inv, eps)
    dzm, dzp = weno5_derivatives(pg, 2, inv, eps)
    uc = (u[:, :, 1:] + u[:, :, :-1]) * 0.5
    vc = (v[:, 1:, :] + v[:, :-1, :]) * 0.5
    wc = (w[1:, :, :] + w[:-1, :, :]) * 0.5
    return _upwind_update(phi, dt, uc, vc, wc, dxm, dxp, dym, dyp, dzm, dzp)


def _face_velocities(axis, ug, vg, wg):
    """Velocity at the faces of component `axis` (ADVECTION_METHOD_3D.h:207-224):
    the component itself and 4-point averages of the other two, read from
    zero-ghosted copies."""
    S = lambda fg, dx_, dy_, dz_, shp: fg[G + dz_:G + dz_ + shp[0], G + dy_:G + dy_ + shp[1], G + dx_:G + dx_ + shp[2]]
    nz, ny, nx = ug.shape[0] - 2 * G, ug.shape[1] - 2 * G, ug.shape[2] - 2 * G - 1
    shp = face_shape((nx, ny, nz), axis)
    if axis == 0:
        uvel = S(ug, 0, 0, 0, shp)
        vvel = (((S(vg, 0, 0, 0, shp) + S(vg, 0, 1, 0, shp)) + S(vg, -1, 0, 0, shp)) + S(vg, -1, 1, 0, shp)) * 0.25
        wvel = (((S(wg, 0, 0, 0, shp) + S(wg, 0, 0, 1, shp)) + S(wg, -1, 0, 0, shp)) + S(wg, -1, 0, 1, shp)) * 0.25
    elif axis == 1:
        uvel = (((S(ug, 0, 0, 0, shp) + S(ug, 1, 0, 0, shp)) + S(ug, 0, -1, 0, shp)) + S(ug, 1, -1, 0, shp)) * 0.25
        vvel = S(vg, 0, 0, 0, shp)
        wvel = (((S(wg, 0, 0, 0, shp) + S(wg, 0, 0, 1, shp)) + S(wg, 0, -1, 0, shp)) + S(wg, 0, -1, 1, shp)) * 0.25
    else:
        uvel = (((S(ug, 0, 0, 0, shp) + S(ug, 1, 0, 0, shp)) + S(ug, 0, 0, -1, shp)) + S(ug, 1, 0, -1, shp)) * 0.25
        vvel = (((S(vg, 0, 0, 0, shp) + S(vg, 0, 1, 0, shp)) + S(vg, 0, 0, -1, shp)) + S(vg, 0, 1, -1, shp)) * 0.25
        wvel = S(wg, 0, 0, 0, shp)
    return uvel, vvel, wvel


def weno5_velocity(u, v, w, dx, dt, eps):
    """Forward-Euler WENO5 self-advection of the three MAC components, every
    face of each component grid (boundary faces included), velocity ghosts
    zero, each component's stencil read from its own zero-ghosted copy.

    The reference's WENO5 velocity call (ADVECTION_3D.h:317-319) passes the
    x-component ghost copy as the stencil source of v and w as well; indexed
    with v's and w's (i, j, k) that copy is read outside its own extent, so
    that call has no well-defined result to reproduce.  The x component,
    which does read its own copy, is identical in both."""
    inv = 1.0 / dx
    ug, vg, wg = zero_ghosts(u), zero_ghosts(v), zero_ghosts(w)
    out = []
    for axis, comp in enumerate((u, v, w)):
        src = (ug, vg, wg)[axis]
        uvel, vvel, wvel = _face_velocities(axis, ug, vg, wg)
        dxm, dxp = weno5_derivatives(src, 0, inv, eps)
        dym, dyp = weno5_derivatives(src, 1, inv, eps)
        dzm, dzp = weno5_derivatives(src, 2, inv, eps)
        out.append(_upwind_update(comp, dt, uvel, vvel, wvel, dxm, dxp, dym, dyp, dzm, dzp))
    return tuple(out)


# ----------------------------------------------------------------------------
# ENO3 (ADVECTION_METHOD_3D.h:1639-1934, the box variant)
# ----------------------------------------------------------------------------

def eno3_derivatives(fg, axis, dx, g=G):
    """One-sided third-order ENO derivatives D-, D+ along `axis` of a
    ghosted field: divided differences of orders 1-3 (the second scaled by
    1/(2dx), the third by (1/dx)/3), each side choosing its stencil by the
    smaller second difference and then the smaller third difference."""
    f = lambda s: _shift(fg, axis, s, g)
    inv = 1.0 / dx
    o2 = 0.5 / dx
    o3 = inv * 1.0 / 3.0
    d1 = {s: inv * (f(s + 1) - f(s)) for s in range(-3, 3)}
    d2 = {s: o2 * (d1[s] - d1[s - 1]) for s in range(-2, 3)}
    d3 = {s: o3 * (d2[s + 1] - d2[s]) for s in range(-2, 2)}
    a = np.abs
    dm = np.where(a(d2[-1]) <= a(d2[0]),
                  np.where(a(d3[-2]) <= a(d3[-1]),
                           (d1[-1] + d2[-1] * dx) + 2.0 * d3[-2] * dx * dx,
                           (d1[-1] + d2[-1] * dx) + 2.0 * d3[-1] * dx * dx),
                  np.where(a(d3[-1]) <= a(d3[0]),
                           (d1[-1] + d2[0] * dx) - d3[-1] * dx * dx,
                           (d1[-1] + d2[0] * dx) - d3[0] * dx * dx))
    dp = np.where(a(d2[0]) <= a(d2[1]),
                  np.where(a(d3[-1]) <= a(d3[0]),
                           (d1[0] - d2[0] * dx) - d3[-1] * dx * dx,
                           (d1[0] - d2[0] * dx) - d3[0] * dx * dx),
                  np.where(a(d3[0]) <= a(d3[1]),
                           (d1[0] - d2[1] * dx) + 2.0 * d3[0] * dx * dx,
                           (d1[0] - d2[1] * dx) + 2.0 * d3[1] * dx * dx))
    return dm, dp


def eno3_velocity(u, v, w, dx, dt):
    """Forward-Euler ENO3 self-advection of the three MAC components
    (ADVECTION_3D.h:323-325: each component with its own zero-ghosted copy,
    the advecting velocity as in the WENO5 path)."""
    ug, vg, wg = zero_ghosts(u), zero_ghosts(v), zero_ghosts(w)
    out = []
    for axis, comp in enumerate((u, v, w)):
        src = (ug, vg, wg)[axis]
        uvel, vvel, wvel = _face_velocities(axis, ug, vg, wg)
        dxm, dxp = eno3_derivatives(src, 0, dx)
        dym, dyp = eno3_derivatives(src, 1, dx)
        dzm, dzp = eno3_derivatives(src, 2, dx)
        out.append(_upwind_update(comp, dt, uvel, vvel, wvel, dxm, dxp, dym, dyp, dzm, dzp))
    return tuple(out)


# ----------------------------------------------------------------------------
# Fast sweeping reinitialisation (LEVELSET_3D.h:601-610, 734-918)
# ----------------------------------------------------------------------------

# The two sweeps of each call, by sweep_direction % 4 (LEVELSET_3D.h:789-818):
# traversal signs (x, y, z) of the first and the second sweep.
FAST_SWEEP_ORDERS = (((1, 1, 1), (-1, -1, -1)), ((-1, 1, -1), (1, -1, 1)),
                     ((1, -1, -1), (-1, 1, 1)), ((-1, -1, 1), (1, 1, -1)))


def fast_sweeping_prepare(phi, dx):
    """The set-up of LEVELSET_3D::FastSweepingMethod (LEVELSET_3D.h:736-781):
    cells farther than 20 dx from the interface and cells with a face
    neighbour of the other sign (ghosts: copies of the boundary cell,
    FillGhostCellsFrom) are fixed; the other cells get +-20 dx.  The
    reference marks neighbours while it scans, but a marked neighbour always
    has a neighbour of the other sign itself, so the fixed set does not
    depend on the scan order.  Returns (phi, fixed)."""
    nb = 20.0 * dx
    g = np.pad(phi, 1, mode="edge")
    pos = g > 0.0
    c = pos[1:-1, 1:-1, 1:-1]
    other = np.zeros(phi.shape, dtype=bool)
    for sl in ((slice(1, -1), slice(1, -1), slice(2, None)), (slice(1, -1), slice(1, -1), slice(0, -2)),
               (slice(1, -1), slice(2, None), slice(1, -1)), (slice(1, -1), slice(0, -2), slice(1, -1)),
               (slice(2, None), slice(1, -1), slice(1, -1)), (slice(0, -2), slice(1, -1), slice(1, -1))):
        other |= pos[sl] != c
    far = np.where(phi > 0, phi, -phi) > nb
    fixed = far | other
    out = np.where(fixed, phi, np.where(phi > 0.0, nb, -nb))
    return out, fixed


def _csqrt(x):
    """C's sqrt: NaN for a negative argument."""
    return math.sqrt(x) if x >= 0.0 else math.nan


def fast_sweep(g, fixed, dx, signs, typo=False):
    """One Gauss-Seidel sweep (LEVELSET_3D.h:837-918) over the interior, z
    outermost and x innermost, in the traversal signs given, in place on the
    ghosted nested list g ([nz+2][ny+2][nx+2]); the ghosts are not touched.

    The reference's INCREASING_SORT3 (MACROS.h:61-68) assigns a3 twice and
    leaves a2 untouched when c < b < a; with `typo` a2 then keeps the value
    of the cell updated before it in the sweep (a2 is a local of Sweep, so
    an input whose first such cell comes before any other update raises:
    the reference reads an uninitialised value there); without it a2 = b."""
    nz, ny, nx = len(g) - 2, len(g[0]) - 2, len(g[0][0]) - 2
    h = dx
    hh = h * h
    hh2 = hh * 2.0
    third = 1.0 / 3.0
    fx = fixed.tolist()
    sx, sy, sz = signs
    a2 = None
    ks = range(nz) if sz > 0 else range(nz - 1, -1, -1)
    js = range(ny) if sy > 0 else range(ny - 1, -1, -1)
    iss = range(nx) if sx > 0 else range(nx - 1, -1, -1)
    for k in ks:
        gk, gkm, gkp = g[k + 1], g[k], g[k + 2]
        for j in js:
            row, rowm, rowp = gk[j + 1], gk[j], gk[j + 2]
            zm, zp = gkm[j + 1], gkp[j + 1]
            fxr = fx[k][j]
            for i in iss:
                if fxr[i]:
                    continue
                pc = row[i + 1]
                if pc > 0.0:
                    l, r = row[i], row[i + 2]
                    a = r if l > r else l
                    l, r = rowm[i + 1], rowp[i + 1]
                    b = r if l > r else l
                    l, r = zm[i + 1], zp[i + 1]
                    c = r if l > r else l
                else:
                    l, r = row[i], row[i + 2]
                    a = l if l > r else r
                    l, r = rowm[i + 1], rowp[i + 1]
                    b = l if l > r else r
                    l, r = zm[i + 1], zp[i + 1]
                    c = l if l > r else r
                if a <= b:
                    if b <= c:
                        a1, a2, a3 = a, b, c
                    elif a <= c:
                        a1, a2, a3 = a, c, b
                    else:
                        a1, a2, a3 = c, a, b
                else:
                    if a <= c:
                        a1, a2, a3 = b, a, c
                    elif b <= c:
                        a1, a2, a3 = b, c, a
                    else:
                        a1, a3 = c, a
                        if typo:
                            if a2 is None:
                                raise ValueError("the reference reads an uninitialised a2 here")
                        else:
                            a2 = b
                if pc > 0.0:
                    upd = a1 + h
                    if upd > a2:
                        d = a1 - a2
                        upd = 0.5 * ((a1 + a2) + _csqrt(hh2 - d * d))
                        if upd > a3:
                            t = (a1 + a2) + a3
                            upd = third * (t + _csqrt(t * t - 3.0 * (((a1 * a1 + a2 * a2) + a3 * a3) - hh)))
                    row[i + 1] = pc if upd > pc else upd
                else:
                    upd = a3 - h
                    if upd < a2:
                        d = a3 - a2
                        upd = 0.5 * ((a3 + a2) - _csqrt(hh2 - d * d))
                        if upd < a1:
                            t = (a1 + a2) + a3
                            upd = third * (t - _csqrt(t * t - 3.0 * (((a1 * a1 + a2 * a2) + a3 * a3) - hh)))
                    row[i + 1] = upd if upd > pc else pc


def fast_sweeping(phi, dx, direction, typo=False, pairs=1):
    """LEVELSET_3D::ReinitializeByFastSweeping on one thread (LEVELSET_3D.h:
    601-610): the set-up, one ghost fill from its result, and the two sweeps
    of sweep_direction % 4 (no ghost fill between them).  `typo`: see
    fast_sweep.

    Every call of the reference starts with the set-up, which resets all
    cells off the interface to +-20 dx, so only the two sweeps of that call
    reach the result, also in FullFastSweepingMethodThreaded's four calls
    (LEVELSET_3D.h:828-835): distances along the six other sweep octants
    are not propagated.  pairs = 4 is the corrected full method: one set-up,
    then the sweep pairs of direction, direction+1, ... (all eight sweeps)."""
    cur, fixed = fast_sweeping_prepare(phi, dx)
    g = np.pad(cur, 1, mode="edge").tolist()
    for p in range(pairs):
        for signs in FAST_SWEEP_ORDERS[(direction + p) % 4]:
            fast_sweep(g, fixed, dx, signs, typo=typo)
    return np.array(g)[1:-1, 1:-1, 1:-1]


# ----------------------------------------------------------------------------
# Sussman reinitialisation (ADVECTION_METHOD_3D.h:745-1637,
# EULERIAN_FLUID_SOLVER_3D.h Reinitialization)
# ----------------------------------------------------------------------------

def sign_function(phi, dx):
    return phi / np.sqrt(phi * phi + dx * dx)


def _godunov_axis(s, dm, dp):
    """Per-axis Godunov selection of the reference's case tree.
    Returns (value, code): code 0 = D-, 1 = D+, 2 = dropped (expansion)."""
    sm, sp = s * dm, s * dp
    both_pos = (sp >= 0) & (sm >= 0)
    both_neg = (sp <= 0) & (sm <= 0) & ~both_pos
    expansion = (sp > 0) & (sm < 0)
    shock = (sp < 0) & (sm > 0)
    with np.errstate(invalid="ignore", divide="ignore"):
        ss = s * (np.abs(dp) - np.abs(dm)) / (dp - dm)
    use_m = both_pos | (shock & (ss > 0))
    use_p = both_neg | (shock & ~(ss > 0))
    code = np.where(use_m, 0, np.where(use_p, 1, 2))
    val = np.where(code == 0, dm, np.where(code == 1, dp, 0.0))
    return val, code, shock


def sussman_step(phi, s, dx, dtau, eps, typo=False, ghost_source=None):
    """One forward-Euler pseudo-step phi - dtau*S*(|grad phi|_G - 1) with the
    sign-preserving clamp (ADVECTION_METHOD_3D.h:1624-1634).

    typo=True reproduces the two leaves of the reference tree that compute
    sqrt(a^2) + b^2 - 1 instead of sqrt(a^2 + b^2) - 1 (x shock, y shock
    resolved to D+, z expansion: ADVECTION_METHOD_3D.h:1463,1605).
    ghost_source: ghosted array to read the stencil from (default: the
    extrapolated copy of phi)."""
    inv = 1.0 / dx
    pg = extrapolate_ghosts(phi) if ghost_source is None else ghost_source
    dxm, dxp = weno5_derivatives(pg, 0, inv, eps)
    dym, dyp = weno5_derivatives(pg, 1, inv, eps)
    dzm, dzp = weno5_derivatives(pg, 2, inv, eps)
    gx, cx, shx = _godunov_axis(s, dxm, dxp)
    gy, cy, shy = _godunov_axis(s, dym, dyp)
    gz, cz, shz = _godunov_axis(s, dzm, dzp)
    mag = np.sqrt((gx * gx + gy * gy) + gz * gz) - 1.0
    if typo:
        bad = shx & shy & (cy == 1) & (cz == 2)
        mag = np.where(bad, (np.sqrt(gx * gx) + gy * gy) - 1.0, mag)
    out = phi - dtau * s * mag
    flip = s * out < 0.0
    out = np.where(flip & (s < 0), -eps, np.where(flip & (s > 0), eps, out))
    return out


def reinitialization_block(phi, dx, iterations, scaling, eps, typo=False):
    """S from the block's input phi, then `iterations` pseudo-steps of
    dtau = dx/scaling, each reading freshly extrapolated ghosts."""
    s = sign_function(phi, dx)
    dtau = dx / scaling
    for _ in range(iterations):
        phi = sussman_step(phi, s, dx, dtau, eps, typo)
    return phi


# ----------------------------------------------------------------------------
# Heaviside, density, viscosity
# ----------------------------------------------------------------------------

def heaviside_projection(phi, e):
    """PROJECTION_3D.h:1452-1470."""
    ooe, oop = 1.0 / e, 1.0 / PI
    mid = (0.5 + phi * ooe * 0.5) + 0.5 * oop * np.sin(PI * phi * ooe)
    return np.where(phi < -e, 0.0, np.where(phi > e, 1.0, mid))


def heaviside_viscosity(phi, e):
    """VISCOSITY_3D.h:1234-1253."""
    ooe, oop = 1.0 / e, 1.0 / PI
    mid = 0.5 * ((1.0 + phi * ooe) + oop * np.sin(PI * phi * ooe))
    return np.where(phi < -e, 0.0, np.where(phi > e, 1.0, mid))


def mix(neg, pos, h):
    """value(phi) = neg + (pos - neg)*H(phi): neg is the phase at phi <= 0."""
    return neg + (pos - neg) * h


# ----------------------------------------------------------------------------
# Pressure projection (PROJECTION_3D.h:416-1449, POISSON_SOLVER_3D.h)
# ----------------------------------------------------------------------------

def divergence(u, v, w, dx, dt):
    """DetermineDivergence (PROJECTION_3D.h:681-722): zero-ghost MAC
    divergence, then scaled by 1/dt."""
    inv = 1.0 / dx
    d = (inv * (u[:, :, 1:] - u[:, :, :-1]) + inv * (v[:, 1:, :] - v[:, :-1, :])) + inv * (w[1:, :, :] - w[:-1, :, :])
    return d * (1.0 / dt)


def face_betas(phi, rho_neg, rho_pos):
    """beta on every MAC face from the sharp cell 1/rho
    (POISSON_SOLVER_3D.h:1080-1085); zero on the box's wall faces."""
    nz, ny, nx = phi.shape
    var = 1.0 / np.where(phi <= 0, rho_neg, rho_pos)
    a = np.abs(phi)

    def beta(vc, vn, ac, an):
        # written as the 'r' arm: vc*vn*(|n|+|c|)/(vn*|c| + vc*|n|)
        with np.errstate(invalid="ignore", divide="ignore"):
            return vc * vn * (an + ac) / (vn * ac + vc * an)

    bx = np.zeros((nz, ny, nx + 1)); by = np.zeros((nz, ny + 1, nx)); bz = np.zeros((nz + 1, ny, nx))
    bx[:, :, 1:-1] = beta(var[:, :, :-1], var[:, :, 1:], a[:, :, :-1], a[:, :, 1:])
    by[:, 1:-1, :] = beta(var[:, :-1, :], var[:, 1:, :], a[:, :-1, :], a[:, 1:, :])
    bz[1:-1, :, :] = beta(var[:-1, :, :], var[1:, :, :], a[:-1, :, :], a[1:, :, :])
    return bx, by, bz, var


def poisson_operator(phi, dx, rho_neg, rho_pos, deflate=True):
    """Matrix-free form of BuildLinearSystemNodeJumpConditionVaribleCoefficient
    (air/water branch, Neumann walls, POISSON_SOLVER_3D.h:1065-1214).

    Row of cell c: diag = inv_dx2 * (sum of beta to full neighbours in the
    order l, r, b, t, d, u), off-diagonal -beta*inv_dx2.  The first cell
    (i=j=k=0) additionally adds the beta of its bottom and down Neumann ghosts
    (the reference's deflation fix, :1145-1179); with the clamped ghost 1/rho
    those betas equal 1/rho of that cell.  A coefficient sum of 0 becomes 1."""
    bx, by, bz, var = face_betas(phi, rho_neg, rho_pos)
    inv2 = 1.0 / (dx * dx)
    coef = ((((bx[:, :, :-1] + bx[:, :, 1:]) + by[:, :-1, :]) + by[:, 1:, :]) + bz[:-1, :, :]) + bz[1:, :, :]
    if deflate:
        # beta to the clamped ghost: var*var*(|g|+|c|)/(var*|c|+var*|g|) with
        # the ghost phi extrapolated; equals var unless both |phi| are 0.
        pg = extrapolate_ghosts(phi, 1)
        c = abs(phi[0, 0, 0]); gb = abs(pg[1, 0, 1]); gd = abs(pg[0, 1, 1]); vv = var[0, 0, 0]
        beta_b = vv * vv * (gb + c) / (vv * gb + vv * c)
        beta_d = vv * vv * (gd + c) / (vv * gd + vv * c)
        coef[0, 0, 0] = (coef[0, 0, 0] + beta_b) + beta_d
    coef = np.where(coef == 0, 1.0, coef)
    return bx * inv2, by * inv2, bz * inv2, inv2 * coef


def apply_poisson(op, p):
    """q = A p in the reference's CSR row order (l, r, b, t, d, u, diag)."""
    ax, ay, az, diag = op
    pg = np.pad(p, 1)
    c = (slice(1, -1),) * 3
    q = np.zeros_like(p)
    q = q + (-ax[:, :, :-1]) * pg[1:-1, 1:-1, :-2]
    q = q + (-ax[:, :, 1:]) * pg[1:-1, 1:-1, 2:]
    q = q + (-ay[:, :-1, :]) * pg[1:-1, :-2, 1:-1]
    q = q + (-ay[:, 1:, :]) * pg[1:-1, 2:, 1:-1]
    q = q + (-az[:-1, :, :]) * pg[:-2, 1:-1, 1:-1]
    q = q + (-az[1:, :, :]) * pg[2:, 1:-1, 1:-1]
    q = q + diag * p
    return q


def poisson_csr(op):
    """The same operator as a CSR matrix in the reference's row numbering
    (k, j, i order) and entry order; used to compare with the reference."""
    ax, ay, az, diag = op
    nz, ny, nx = diag.shape
    vals, cols, rowptr = [], [], [0]
    idx = lambda i, j, k: i + nx * (j + ny * k)
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                for (cond, val, col) in ((i > 0, ax[k, j, i], (i - 1, j, k)), (i < nx - 1, ax[k, j, i + 1], (i + 1, j, k)),
                                         (j > 0, ay[k, j, i], (i, j - 1, k)), (j < ny - 1, ay[k, j + 1, i], (i, j + 1, k)),
                                         (k > 0, az[k, j, i], (i, j, k - 1)), (k < nz - 1, az[k + 1, j, i], (i, j, k + 1))):
                    if cond:
                        vals.append(-val); cols.append(idx(*col))
                vals.append(diag[k, j, i]); cols.append(idx(i, j, k))
                rowptr.append(len(vals))
    return np.array(vals), np.array(cols, dtype=np.int32), np.array(rowptr, dtype=np.int32)


def pcg(apply_A, diag, b, x0, tol, max_iter, criterion="abs"):
    """Jacobi-PCG of PCG_METHOD.cpp:4-126.

    criterion "abs": stop when r.z < tol^2 (the reference's test, :87).
    criterion "rel": stop when ||r||_2 / ||b||_2 < tol.
    Returns (x, iterations, final r.z, final relative residual)."""
    x = x0.copy()
    r = b - apply_A(x)
    p = r / diag
    rz = _seqdot(r, p)
    bb = _seqdot(b, b)
    bnorm = math.sqrt(bb) or 1.0
    it = 0
    if criterion != "abs" and (bb == 0.0 or math.sqrt(_seqdot(r, r)) / bnorm <= tol):
        return x, 0, rz, math.sqrt(_seqdot(r, r)) / bnorm
    while it < max_iter:
        q = apply_A(p)
        alpha = rz / _seqdot(p, q)
        x = x + alpha * p
        r = r - alpha * q
        s = r / diag
        rz_old = rz
        rz = _seqdot(r, s)
        if criterion == "abs":
            if rz < tol * tol:
                break
        elif math.sqrt(_seqdot(r, r)) / bnorm < tol:
            break
        beta = rz / rz_old
        p = p * beta + s
        it += 1
    return x, it, rz, math.sqrt(_seqdot(r, r)) / bnorm


# ----------------------------------------------------------------------------
# Surface tension (LEVELSET_3D.h:963-1082, PROJECTION_3D.h:746-792,
# POISSON_SOLVER_3D.h:1216-1328, EULERIAN_FLUID_SOLVER_3D.h:2741-2745)
# ----------------------------------------------------------------------------

def curvature(phi, dx, typo=False):
    """LEVELSET_3D::ComputeCurvatures (curvature_by_levelset): kappa from
    central differences of the level set with one layer of linearly
    extrapolated ghosts,
      kappa = -(px^2 pyy - 2 px py pxy + py^2 pxx + px^2 pzz - 2 px pz pxz
                + pz^2 pxx + py^2 pzz - 2 py pz pyz + pz^2 pyy) / |grad phi|^3,
    clamped from below at -1/dx (:1061-1068).  typo=True reproduces the
    reference's two slips: the factor 2 missing on the py pz pyz term
    (:1033) and, in the zero-gradient fallback of one-sided differences, the
    z difference multiplied by dz instead of divided (:1037).  Where even the
    fallback gradient is zero the reference exits the process (:1040-1044);
    kappa is 0 there.  Returns (kappa, max |kappa| over cells with |phi| < 0.1)."""
    a = extrapolate_ghosts(phi, 1)
    nz, ny, nx = phi.shape

    def at(di, dj, dk):
        return a[1 + dk:1 + dk + nz, 1 + dj:1 + dj + ny, 1 + di:1 + di + nx]

    inv = 1.0 / dx
    o2 = 0.5 / dx
    o2sq = 1.0 / (dx * dx)
    c = at(0, 0, 0)
    px = (at(1, 0, 0) - at(-1, 0, 0)) * o2
    py = (at(0, 1, 0) - at(0, -1, 0)) * o2
    pz = (at(0, 0, 1) - at(0, 0, -1)) * o2
    pxx = ((at(1, 0, 0) - 2 * c) + at(-1, 0, 0)) * o2sq
    pyy = ((at(0, 1, 0) - 2 * c) + at(0, -1, 0)) * o2sq
    pzz = ((at(0, 0, 1) - 2 * c) + at(0, 0, -1)) * o2sq
    pxy = ((((at(1, 1, 0) - at(1, -1, 0)) - at(-1, 1, 0)) + at(-1, -1, 0)) * o2) * o2
    pxz = ((((at(1, 0, 1) - at(1, 0, -1)) - at(-1, 0, 1)) + at(-1, 0, -1)) * o2) * o2
    pyz = ((((at(0, 1, 1) - at(0, 1, -1)) - at(0, -1, 1)) + at(0, -1, -1)) * o2) * o2

    def num(px, py, pz):
        t = px * px * pyy - 2.0 * px * py * pxy
        t = t + py * py * pxx
        t = t + px * px * pzz
        t = t - 2.0 * px * pz * pxz
        t = t + pz * pz * pxx
        t = t + py * py * pzz
        t = t - (py * pz * pyz if typo else 2.0 * py * pz * pyz)
        return t + pz * pz * pyy

    mag = np.sqrt((px * px + py * py) + pz * pz)
    deno = mag * mag * mag
    with np.errstate(divide="ignore", invalid="ignore"):
        curv = -num(px, py, pz) * (1.0 / deno)
        # fallback: one-sided differences where the central gradient vanishes
        fx = (at(1, 0, 0) - c) * inv
        fy = (at(0, 1, 0) - c) * inv
        fz = (at(0, 0, 1) - c) * (dx if typo else inv)
        fm = np.sqrt((fx * fx + fy * fy) + fz * fz)
        fd = fm * fm * fm
        fcurv = np.where(fd != 0, -num(fx, fy, fz) * (1.0 / fd), 0.0)
    curv = np.where(deno != 0, curv, fcurv)
    tol = 1.0 / dx
    kappa = np.where(curv < -tol, -tol, curv)
    band = np.abs(phi) < 1e-1
    kmax = float(np.max(np.abs(kappa[band]))) if band.any() else 0.0
    return kappa, kmax


def jump_rhs(phi, jc, dx, rho_neg, rho_pos, walls=True):
    """Sum over the six arms of the ghost-fluid jump terms F of the pressure
    right-hand side b = -div - F_X - F_Y - F_Z (POISSON_SOLVER_3D.h:1216-1328)
    with jc_on_derivative = 0: an arm whose two cells lie in different phases
    carries F = +-inv_dx2 * a * beta, a = (jc_c |phi_n| + jc_n |phi_c|) /
    (|phi_c| + |phi_n|), + when the cell is in the phi <= 0 phase.  With
    walls (the reference), arms to the wall ghosts are evaluated too, with the
    ghost phi the reference holds when it builds the system: ComputeNormals
    (LEVELSET_3D.h:931), called just before, fills the ghosts by copying the
    nearest cell, so a wall arm never crosses the interface.  Without
    (corrected), only arms between two cells of the box are evaluated, as
    only they have a face the velocity update corrects.  Both give the same
    terms.  Returns (F_X, F_Y, F_Z)."""
    pg = np.pad(phi, 1, mode="edge")
    var = 1.0 / np.where(phi <= 0, rho_neg, rho_pos)
    vg = np.pad(var, 1, mode="edge")
    jg = np.pad(jc, 1)
    nz, ny, nx = phi.shape
    inv2 = 1.0 / (dx * dx)

    def nb(arr, di, dj, dk):
        return arr[1 + dk:1 + dk + nz, 1 + dj:1 + dj + ny, 1 + di:1 + di + nx]

    pc, vc, jcc = phi, var, jc
    ac = np.abs(pc)
    out = []
    for (lo, hi) in (((-1, 0, 0), (1, 0, 0)), ((0, -1, 0), (0, 1, 0)), ((0, 0, -1), (0, 0, 1))):
        F = []
        for d, low in ((lo, True), (hi, False)):
            pn, vn, jn = nb(pg, *d), nb(vg, *d), nb(jg, *d)
            an = np.abs(pn)
            with np.errstate(divide="ignore", invalid="ignore"):
                a = (jcc * an + jn * ac) / (ac + an)
                if low:   # l, b, d arms
                    beta = vc * vn * (an + ac) / (vc * an + vn * ac)
                else:     # r, t, u arms
                    beta = vc * vn * (an + ac) / (vn * ac + vc * an)
            f = np.where((pc <= 0) & (pn > 0), inv2 * a * beta,
                         np.where((pc > 0) & (pn <= 0), -inv2 * a * beta, 0.0))
            if not walls:
                ax = 2 - [i for i in range(3) if d[i] != 0][0]
                sl = [slice(None)] * 3
                sl[ax] = 0 if low else -1
                f = f.copy()
                f[tuple(sl)] = 0.0
            F.append(f)
        out.append(F[0] + F[1])
    return tuple(out)


def velocity_correction(u, v, w, p, phi, dx, dt, rho_neg, rho_pos, mode="corrected", jc=None):
    """UpdateVelocityByPressureGradientVariableDensity (PROJECTION_3D.h:1099-1449).

    faithful (the reference as it runs): same-side faces u -= dt*(p_c -
    p_nb)/rho_c/dx with the sharp rho of the cell on the face's + side; faces
    whose two cells have phi_c*phi_nb <= 0: u -= dt*(p_c - p_nb -/+ jump)/
    rho_f/dx with rho_f the smeared density (PROJECTION_3D Heaviside, eps =
    1.5 dx) of the face-averaged phi.  Only w is updated (the u and v branches
    of the reference are gated on pipe-mode flags, :1188,1211,1297,1320) and
    the bottom face of the first cell is updated against a zero ghost
    pressure (bc*bc_d >= 0 holds for row index 0).

    corrected: u, v and w updated, wall faces untouched, every interior face
    with the pressure matrix's own coefficient, u -= dt*beta_f*(p_c - p_nb
    -/+ jump)/dx (beta_f of POISSON_SOLVER_3D.h:1080-1085 as face_betas
    computes it; the jump on faces whose cells lie in different phases, - when
    the cell on the face's + side has phi > 0).  This is the gradient the
    matrix was built from, so the corrected velocity is divergence free to
    the solve's residual, the interface included."""
    nz, ny, nx = phi.shape
    rho_c = np.where(phi <= 0, rho_neg, rho_pos)
    pg = extrapolate_ghosts(phi, 1)
    jc = np.zeros_like(phi) if jc is None else jc
    e = 1.5 * dx
    inv = 1.0 / dx
    out = [u.copy(), v.copy(), w.copy()]
    if mode != "faithful":
        betas = face_betas(phi, rho_neg, rho_pos)[:3]
        for axis in (0, 1, 2):
            ax = 2 - axis
            sl_c = [slice(None)] * 3; sl_n = [slice(None)] * 3
            sl_c[ax] = slice(1, None); sl_n[ax] = slice(0, -1)
            sl_c, sl_n = tuple(sl_c), tuple(sl_n)
            ph_c, ph_n = phi[sl_c], phi[sl_n]
            fs = [slice(None)] * 3
            fs[ax] = slice(1, -1)
            fs = tuple(fs)
            beta = betas[axis][fs]
            dp = p[sl_c] - p[sl_n]
            with np.errstate(invalid="ignore", divide="ignore"):
                jump = (jc[sl_c] * np.abs(ph_n) + jc[sl_n] * np.abs(ph_c)) / (np.abs(ph_n) + np.abs(ph_c))
            cross = (ph_c <= 0) != (ph_n <= 0)
            dp = np.where(cross, np.where(ph_c <= 0, dp + jump, dp - jump), dp)
            f = out[axis]
            f[fs] = f[fs] - dt * dp * beta * inv
        return tuple(out)
    for axis in (2,):
        ax = 2 - axis
        sl_c = [slice(None)] * 3; sl_n = [slice(None)] * 3
        sl_c[ax] = slice(1, None); sl_n[ax] = slice(0, -1)
        sl_c, sl_n = tuple(sl_c), tuple(sl_n)
        ph_c, ph_n = phi[sl_c], phi[sl_n]
        # face phi from the extrapolated ghost copy (interior faces only here)
        face_phi = 0.5 * (ph_c + ph_n)
        rho_f = mix(rho_neg, rho_pos, heaviside_projection(face_phi, e))
        inv_rho_f = 1.0 / rho_f
        inv_rho_c = 1.0 / rho_c[sl_c]
        with np.errstate(invalid="ignore", divide="ignore"):
            jump = (jc[sl_c] * np.abs(ph_n) + jc[sl_n] * np.abs(ph_c)) / (np.abs(ph_n) + np.abs(ph_c))
        dp = p[sl_c] - p[sl_n]
        same = ph_c * ph_n > 0
        upd_same = dt * dp * inv_rho_c * inv
        upd_neg = dt * (dp + jump) * inv_rho_f * inv
        upd_pos = dt * (dp - jump) * inv_rho_f * inv
        upd = np.where(same, upd_same, np.where(ph_c <= 0, upd_neg, upd_pos))
        f = out[axis]
        fs = [slice(None)] * 3
        fs[ax] = slice(1, -1)
        f[tuple(fs)] = f[tuple(fs)] - upd
        # the first cell's bottom face against the zero ghost pressure
        c = phi[0, 0, 0]; g = pg[0, 1, 1]
        fphi = 0.5 * (c + g)
        if c * g > 0:
            f[0, 0, 0] = f[0, 0, 0] - dt * (p[0, 0, 0] - 0.0) * (1.0 / rho_c[0, 0, 0]) * inv
        else:
            rf = mix(rho_neg, rho_pos, heaviside_projection(np.array(fphi), e))
            # the ghost jump condition is 0 (jc_on_solution is zero outside the box)
            jmp = (jc[0, 0, 0] * abs(g) + 0.0 * abs(c)) / (abs(g) + abs(c))
            if c <= 0:
                f[0, 0, 0] = f[0, 0, 0] - dt * (p[0, 0, 0] - 0.0 + jmp) * (1.0 / rf) * inv
            else:
                f[0, 0, 0] = f[0, 0, 0] - dt * (p[0, 0, 0] - 0.0 - jmp) * (1.0 / rf) * inv
    return tuple(out)


def projection(phi, u, v, w, dx, dt, rho_neg, rho_pos, tol, max_iter, mode="corrected", criterion="abs", p0=None,
               sigma=0.0, curvature_typo=False):
    """PROJECTION_3D::Solve for the air/water box with Neumann walls:
    divergence, jump condition jc = sigma*kappa (DetermineJumpConditionField,
    PROJECTION_3D.h:746-792), operator, RHS = -div - F (jump terms) minus its
    mean (POISSON_SOLVER_3D.h:225-246), Jacobi-PCG, velocity correction with
    the jump.  Returns (u, v, w, p, info)."""
    div = divergence(u, v, w, dx, dt)
    # faithful: the reference's deflated (nonsingular) system; corrected: the
    # singular consistent Neumann system, so that the corrected velocity's
    # divergence is the residual in every cell (the deflation would leave the
    # residual's sum in the first cell)
    op = poisson_operator(phi, dx, rho_neg, rho_pos, deflate=(mode == "faithful"))
    jc = None
    if sigma != 0.0:
        kappa, _ = curvature(phi, dx, curvature_typo)
        jc = sigma * kappa
        FX, FY, FZ = jump_rhs(phi, jc, dx, rho_neg, rho_pos, walls=(mode == "faithful"))
        b = ((-div - FX) - FY) - FZ
    else:
        b = -div
    b = b - (1.0 / b.size) * _seqsum(b)
    x0 = np.zeros_like(b) if p0 is None else p0
    p, it, rz, rel = pcg(lambda x: apply_poisson(op, x), op[3], b, x0, tol, max_iter, criterion)
    u2, v2, w2 = velocity_correction(u, v, w, p, phi, dx, dt, rho_neg, rho_pos, mode, jc=jc)
    return u2, v2, w2, p, {"iterations": it, "rz": rz, "rel_residual": rel, "b": b, "op": op, "jc": jc}


# ----------------------------------------------------------------------------
# Viscosity (VISCOSITY_3D.h)
# ----------------------------------------------------------------------------

def _cell_ghost(phi):
    return extrapolate_ghosts(phi, 1)


def viscosity_samples(phi, axis):
    """Level-set samples used by the viscous coefficients of component
    `axis` (VISCOSITY_3D.h:462-470 for x, 502-510 for y, 541-549 for z):
    face average (density), the two cells across the face (normal stress)
    and four edge averages (shear), from a 1-layer extrapolated ghost copy."""
    pg = _cell_ghost(phi)
    nz, ny, nx = phi.shape
    shp = face_shape((nx, ny, nz), axis)

    def P(di, dj, dk):
        return pg[1 + dk:1 + dk + shp[0], 1 + dj:1 + dj + shp[1], 1 + di:1 + di + shp[2]]

    if axis == 0:
        half = 0.5 * (P(-1, 0, 0) + P(0, 0, 0))
        n_hi, n_lo = P(0, 0, 0), P(-1, 0, 0)
        e1 = 0.25 * (((P(-1, 0, 0) + P(0, 0, 0)) + P(-1, 1, 0)) + P(0, 1, 0))   # cu
        e2 = 0.25 * (((P(-1, 0, 0) + P(0, 0, 0)) + P(-1, -1, 0)) + P(0, -1, 0))  # cd
        e3 = 0.25 * (((P(-1, 0, 0) + P(0, 0, 0)) + P(-1, 0, 1)) + P(0, 0, 1))   # ct
        e4 = 0.25 * (((P(-1, 0, 0) + P(0, 0, 0)) + P(-1, 0, -1)) + P(0, 0, -1))  # cb
    elif axis == 1:
        half = 0.5 * (P(0, -1, 0) + P(0, 0, 0))
        n_hi, n_lo = P(0, 0, 0), P(0, -1, 0)
        e1 = 0.25 * (((P(0, -1, 0) + P(1, -1, 0)) + P(0, 0, 0)) + P(1, 0, 0))   # cu (x+)
        e2 = 0.25 * (((P(-1, -1, 0) + P(0, -1, 0)) + P(-1, 0, 0)) + P(0, 0, 0))  # cl (x-)
        e3 = 0.25 * (((P(0, -1, 1) + P(0, -1, 0)) + P(0, 0, 1)) + P(0, 0, 0))   # ct
        e4 = 0.25 * (((P(0, -1, -1) + P(0, -1, 0)) + P(0, 0, -1)) + P(0, 0, 0))  # cb
    else:
        half = 0.5 * (P(0, 0, -1) + P(0, 0, 0))
        n_hi, n_lo = P(0, 0, 0), P(0, 0, -1)
        e1 = 0.25 * (((P(0, 0, -1) + P(1, 0, -1)) + P(0, 0, 0)) + P(1, 0, 0))   # ct (x+)
        e2 = 0.25 * (((P(0, 0, -1) + P(-1, 0, -1)) + P(0, 0, 0)) + P(-1, 0, 0))  # cb (x-)
        e3 = 0.25 * (((P(0, 0, -1) + P(0, 1, -1)) + P(0, 0, 0)) + P(0, 1, 0))   # cu (y+)
        e4 = 0.25 * (((P(0, 0, -1) + P(0, -1, -1)) + P(0, 0, 0)) + P(0, -1, 0))  # cd (y-)
    return half, n_hi, n_lo, e1, e2, e3, e4


DIRECTIONS = ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1))


def semi_implicit_coefficients(phi, axis, dx, dt, rho_neg, rho_pos, mu_neg, mu_pos):
    """Coefficients of the semi-implicit system of component `axis`, in the
    direction order of the reference's builder (coef_1..coef_6 = +x, -x, +y,
    -y, +z, -z; POISSON_SOLVER_3D.h:3383-3411): 2 dt mu/rho_f on the two
    normal arms, dt mu/rho_f on the tangential arms (VISCOSITY_3D.h:603-611,
    744-749, 811-816, Re = 1).  mu on the normal arms is sampled at the two
    cells across the face, on the tangential arms at the four-cell edge
    averages; rho_f from the face-averaged phi.
    Returns (coefs[6], rho_f, [mu_hi, mu_lo, mu_t1+, mu_t1-, mu_t2+, mu_t2-])."""
    e = 1.5 * dx
    half, n_hi, n_lo, e1, e2, e3, e4 = viscosity_samples(phi, axis)
    rho_f = mix(rho_neg, rho_pos, heaviside_viscosity(half, e))
    mu = [mix(mu_neg, mu_pos, heaviside_viscosity(a, e)) for a in (n_hi, n_lo, e1, e2, e3, e4)]
    two = 2.0 * dt / (1.0 * rho_f)
    one = dt / (1.0 * rho_f)
    t1, t2 = [a for a in (0, 1, 2) if a != axis]
    c = [None] * 6
    c[2 * axis], c[2 * axis + 1] = two * mu[0], two * mu[1]
    c[2 * t1], c[2 * t1 + 1] = one * mu[2], one * mu[3]
    c[2 * t2], c[2 * t2 + 1] = one * mu[4], one * mu[5]
    return c, rho_f, mu


def semi_implicit_explicit_term(u, v, w, axis, dx, dt, rho_f, mu):
    """u* + dt/rho_f * (transpose stress terms), VISCOSITY_3D.h:620-630
    (x component; y and z by the same pattern), zero velocity ghosts."""
    inv = 1.0 / dx
    vel = (u, v, w)
    g = [zero_ghosts(a, 1) for a in vel]
    shp = vel[axis].shape

    def F(comp, di, dj, dk):
        a = g[comp]
        return a[1 + dk:1 + dk + shp[0], 1 + dj:1 + dj + shp[1], 1 + di:1 + di + shp[2]]

    off = {0: (1, 0, 0), 1: (0, 1, 0), 2: (0, 0, 1)}
    others = [a for a in (0, 1, 2) if a != axis]
    total = vel[axis]
    coef = dt / (1.0 * rho_f)
    for n, t in enumerate(others):
        mu_p, mu_m = mu[2 + 2 * n], mu[3 + 2 * n]
        ot = off[t]; oa = off[axis]
        # d/dt( mu * d(vel_t)/d(axis) ) at the face of component `axis`
        hi = mu_p * inv * (F(t, ot[0], ot[1], ot[2]) - F(t, ot[0] - oa[0], ot[1] - oa[1], ot[2] - oa[2]))
        lo = mu_m * inv * (F(t, 0, 0, 0) - F(t, -oa[0], -oa[1], -oa[2]))
        total = total + coef * (inv * (hi - lo))
    return total


def semi_implicit_system(coef, explicit_term, comp0, axis, inv2, unknown, dval):
    """Assemble the semi-implicit system for one component in the
    reference's row order (k, j, i over unknowns) and entry order
    (-x, +x, -y, +y, -z, +z, diagonal).  Returns a dense operator closure,
    the Jacobi diagonal, the RHS and the unknown index map."""
    shp = comp0.shape
    # entry order of the reference's rows: -x, +x, -y, +y, -z, +z
    dirs = [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]
    arm_of = {o: n for n, o in enumerate(DIRECTIONS)}
    ug = np.pad(unknown, 1)
    dg = np.pad(dval, 1)
    coef_sum = np.zeros(shp)
    rhs = explicit_term.copy()
    nb_coef = []
    for d in dirs:
        c = coef[arm_of[d]] * 1.0
        m = ug[1 + d[2]:1 + d[2] + shp[0], 1 + d[1]:1 + d[1] + shp[1], 1 + d[0]:1 + d[0] + shp[2]]
        coef_sum = coef_sum + np.where(m, c, 0.0)
        nb_coef.append((d, np.where(m, -c * inv2, 0.0), m))
    for d in dirs:
        c = coef[arm_of[d]]
        m = ug[1 + d[2]:1 + d[2] + shp[0], 1 + d[1]:1 + d[1] + shp[1], 1 + d[0]:1 + d[0] + shp[2]]
        coef_sum = coef_sum + np.where(~m, c, 0.0)
    coef_sum = np.where(coef_sum == 0, 1.0, coef_sum)
    diag = 1.0 + inv2 * coef_sum
    for d in dirs:
        c = coef[arm_of[d]]
        m = ug[1 + d[2]:1 + d[2] + shp[0], 1 + d[1]:1 + d[1] + shp[1], 1 + d[0]:1 + d[0] + shp[2]]
        val = dg[1 + d[2]:1 + d[2] + shp[0], 1 + d[1]:1 + d[1] + shp[1], 1 + d[0]:1 + d[0] + shp[2]]
        rhs = rhs + np.where(~m, c * inv2 * val, 0.0)

    def apply(x):
        xg = np.pad(np.where(unknown, x, 0.0), 1)
        q = np.zeros(shp)
        for d, a, m in nb_coef:
            q = q + a * xg[1 + d[2]:1 + d[2] + shp[0], 1 + d[1]:1 + d[1] + shp[1], 1 + d[0]:1 + d[0] + shp[2]]
        q = q + diag * x
        return np.where(unknown, q, 0.0)

    return apply, np.where(unknown, diag, 1.0), np.where(unknown, rhs, 0.0)


def solve_semi_implicit(comp0, coef, explicit_term, axis, dx, tol, max_iter, unknown=None, dval=None,
                        criterion="abs", x0=None):
    """Jacobi-PCG on the semi-implicit system of one component (the reference
    solves it with the projection's PCG, VISCOSITY_3D.h:711)."""
    shp = comp0.shape
    unknown = np.ones(shp, dtype=bool) if unknown is None else unknown
    dval = np.zeros(shp) if dval is None else dval
    inv2 = 1.0 / (dx * dx)
    apply, diag, rhs = semi_implicit_system(coef, explicit_term, comp0, axis, inv2, unknown, dval)
    start = np.where(unknown, comp0 if x0 is None else x0, 0.0)
    x, it, rz, rel = pcg(apply, diag, rhs, start, tol, max_iter, criterion)
    return np.where(unknown, x, dval), it, rel


def wall_normal_mask(n, axis):
    """Unknown faces of component `axis` in the box: all but the two wall
    planes normal to the axis."""
    shp = face_shape(n, axis)
    m = np.ones(shp, dtype=bool)
    ax = 2 - axis
    sl = [slice(None)] * 3
    sl[ax] = 0; m[tuple(sl)] = False
    sl[ax] = -1; m[tuple(sl)] = False
    return m


def viscosity_semi_implicit(phi, u, v, w, dx, dt, rho_neg, rho_pos, mu_neg, mu_pos, tol, max_iter, criterion="rel"):
    """Semi-implicit viscosity for the box: per component, implicit in
    d/dx_j(mu du_i/dx_j) (factor 2 on the normal arm), explicit transpose
    terms; wall-normal faces are held at zero, tangential ghosts are zero."""
    nx = phi.shape[2]; ny = phi.shape[1]; nz = phi.shape[0]
    n = (nx, ny, nz)
    out, iters = [], []
    comps = (u, v, w)
    for axis in range(3):
        coef, rho_f, mu = semi_implicit_coefficients(phi, axis, dx, dt, rho_neg, rho_pos, mu_neg, mu_pos)
        ex = semi_implicit_explicit_term(u, v, w, axis, dx, dt, rho_f, mu)
        mask = wall_normal_mask(n, axis)
        x, it, _ = solve_semi_implicit(comps[axis], coef, ex, axis, dx, tol, max_iter, mask, None, criterion)
        out.append(np.where(mask, x, 0.0)); iters.append(it)
    return tuple(out), iters


def _explicit_face_update(axis, vel, rho_h, mu, dx, dt, faces, faithful):
    """Explicit viscous increment of component `axis` on the faces listed in
    `faces` (index arrays (k, j, i) into that component's array), from the
    zero-ghosted velocities `vel` (each padded by one layer).

    faithful: the expressions of VISCOSITY_3D.h:482-486 (x), 521-525 (y),
    560-564 (z), operand for operand, including their velocity indices: the
    y update reads w at (i,j,k) and (i,j-1,k) on its z+ edge and one level
    lower on its z- edge, and the z update reads u at i (not i+1) on its x+
    edge and v at j (not j+1) on its y+ edge.  corrected: the same
    discretisation with every transposed-stress term on its own edge, as the
    x update has it."""
    K, J, I = faces
    inv = 1.0 / dx
    g = [vel[0], vel[1], vel[2]]

    def at(comp, di, dj, dk):
        return g[comp][K + 1 + dk, J + 1 + dj, I + 1 + di]

    rh = rho_h[K, J, I]
    m = [a[K, J, I] for a in mu]  # hi, lo, e1, e2, e3, e4 (viscosity_samples order)
    coef = dt * (1.0 / rh)
    if axis == 0:
        u = at(0, 0, 0, 0)
        first = 2.0 * coef * inv * (m[0] * inv * (at(0, 1, 0, 0) - u) - m[1] * inv * (u - at(0, -1, 0, 0)))
        second = coef * inv * (m[2] * (inv * (at(0, 0, 1, 0) - u) + inv * (at(1, 0, 1, 0) - at(1, -1, 1, 0)))
                               - m[3] * (inv * (u - at(0, 0, -1, 0)) + inv * (at(1, 0, 0, 0) - at(1, -1, 0, 0))))
        third = coef * inv * (m[4] * (inv * (at(0, 0, 0, 1) - u) + inv * (at(2, 0, 0, 1) - at(2, -1, 0, 1)))
                              - m[5] * (inv * (u - at(0, 0, 0, -1)) + inv * (at(2, 0, 0, 0) - at(2, -1, 0, 0))))
        return u + ((first + second) + third)
    if axis == 1:
        v = at(1, 0, 0, 0)
        first = coef * inv * (m[2] * (inv * (at(0, 1, 0, 0) - at(0, 1, -1, 0)) + inv * (at(1, 1, 0, 0) - v))
                              - m[3] * (inv * (at(0, 0, 0, 0) - at(0, 0, -1, 0)) + inv * (v - at(1, -1, 0, 0))))
        second = 2.0 * coef * inv * (m[0] * inv * (at(1, 0, 1, 0) - v) - m[1] * inv * (v - at(1, 0, -1, 0)))
        zt = 0 if faithful else 1  # the w level of the z+ edge
        third = coef * inv * (m[4] * (inv * (at(1, 0, 0, 1) - v) + inv * (at(2, 0, 0, zt) - at(2, 0, -1, zt)))
                              - m[5] * (inv * (v - at(1, 0, 0, -1)) + inv * (at(2, 0, 0, zt - 1) - at(2, 0, -1, zt - 1))))
        return v + ((first + second) + third)
    w = at(2, 0, 0, 0)
    xt = 0 if faithful else 1  # the u column of the x+ edge
    yt = 0 if faithful else 1  # the v row of the y+ edge
    first = coef * inv * (m[2] * (inv * (at(0, xt, 0, 0) - at(0, xt, 0, -1)) + inv * (at(2, 1, 0, 0) - w))
                          - m[3] * (inv * (at(0, xt - 1, 0, 0) - at(0, xt - 1, 0, -1)) + inv * (w - at(2, -1, 0, 0))))
    second = coef * inv * (m[4] * (inv * (at(1, 0, yt, 0) - at(1, 0, yt, -1)) + inv * (at(2, 0, 1, 0) - w))
                           - m[5] * (inv * (at(1, 0, yt - 1, 0) - at(1, 0, yt - 1, -1)) + inv * (w - at(2, 0, -1, 0))))
    third = 2.0 * coef * inv * (m[0] * inv * (at(2, 0, 0, 1) - w) - m[1] * inv * (w - at(2, 0, 0, -1)))
    return w + ((first + second) + third)


def explicit_viscosity(phi, u, v, w, dx, dt, rho_neg, rho_pos, mu_neg, mu_pos, faithful=False):
    """The air/water viscosity of VISCOSITY_3D::ApplyViscosity
    (VISCOSITY_3D.h:452-563): an explicit variable-viscosity stress update
    with the smeared density of the face-averaged phi and the smeared
    viscosity at the two cells across the face (normal stress) and at the
    four edge averages (shear), Heaviside eps = 1.5 dx
    (EULERIAN_FLUID_SOLVER_3D.h:394, VISCOSITY_3D.h:1234-1253).  Velocity
    ghosts are zero; phi has one layer of linearly extrapolated ghosts.

    faithful (the reference as it runs, one thread): x, then y, then z, each
    updated in place in (k, j, i) order, so a face reads the already updated
    x-1, y-1, z-1 neighbours of its own component and later components read
    the earlier ones' new values; every face of the component is updated,
    the wall faces included; the velocity indices of _explicit_face_update.
    The in-place order is evaluated here by hyperplanes i+j+k = s (a face
    depends on its own component only through hyperplane s-1), which reads
    exactly what the sequential loop reads.

    corrected: one explicit Euler step of the stress divergence from the
    input velocities (no in-place order), transposed terms on their own
    edges, wall-normal faces left as they are (no penetration)."""
    nz, ny, nx = phi.shape
    n = (nx, ny, nz)
    e = 1.5 * dx
    out = [np.array(u, dtype=float), np.array(v, dtype=float), np.array(w, dtype=float)]
    src = [np.pad(a, 1) for a in out]
    for axis in range(3):
        half, n_hi, n_lo, e1, e2, e3, e4 = viscosity_samples(phi, axis)
        rho_h = mix(rho_neg, rho_pos, heaviside_viscosity(half, e))
        mu = [mix(mu_neg, mu_pos, heaviside_viscosity(a, e)) for a in (n_hi, n_lo, e1, e2, e3, e4)]
        shp = face_shape(n, axis)
        Kg, Jg, Ig = np.indices(shp)
        if faithful:
            vel = [np.pad(a, 1) for a in out]  # current values, earlier components updated
            s_of = Kg + Jg + Ig
            for s_ in range(int(s_of.max()) + 1):
                sel = s_of == s_
                faces = (Kg[sel], Jg[sel], Ig[sel])
                vel[axis][faces[0] + 1, faces[1] + 1, faces[2] + 1] = _explicit_face_update(
                    axis, vel, rho_h, mu, dx, dt, faces, True)
            out[axis] = vel[axis][1:-1, 1:-1, 1:-1].copy()
        else:
            ax = 2 - axis
            keep = (Kg, Jg, Ig)[ax]
            inner = (keep > 0) & (keep < shp[ax] - 1)
            faces = (Kg[inner], Jg[inner], Ig[inner])
            res = out[axis].copy()
            res[faces] = _explicit_face_update(axis, src, rho_h, mu, dx, dt, faces, False)
            out[axis] = res
    return tuple(out)


# ----------------------------------------------------------------------------
# CFL (EULERIAN_FLUID_SOLVER_3D.h:2673-2785)
# ----------------------------------------------------------------------------

def cfl_dt(u, v, w, dx, gravity_y, nu_max=0.0, surface_term=0.0):
    """1/cfl with cfl = 0.5*(c + v + sqrt((c+v)^2 + 4 g^2 + 4 s^2));
    c = sum max|u_d|/dx, g = sqrt(|g_y|/dx), v = nu_max*6/dx^2 when the
    viscosity is explicit (0 when semi-implicit)."""
    inv = 1.0 / dx
    c_f = (np.max(np.abs(u)) * inv + np.max(np.abs(v)) * inv) + np.max(np.abs(w)) * inv
    g_f = math.sqrt(abs(gravity_y) * inv)
    inv2 = 1.0 / (dx * dx)
    v_f = nu_max * ((2.0 * inv2 + 2.0 * inv2) + 2.0 * inv2)
    s_f = surface_term
    cv = c_f + v_f
    cfl = 0.5 * (cv + math.sqrt((cv * cv + 4.0 * (g_f * g_f)) + 4.0 * (s_f * s_f)))
    return 1.0 / cfl


# ----------------------------------------------------------------------------
# Whole timestep, corrected specification (the GPU path's contract)
# ----------------------------------------------------------------------------

def add_gravity(u, v, w, g, dt):
    """u_d += dt*g_d on every face except the two wall planes normal to d
    (ApplyGravity, EULERIAN_FLUID_SOLVER_3D.h:2237-2269; wall faces hold the
    no-penetration zero)."""
    out = []
    for axis, f in enumerate((u, v, w)):
        f = f.copy()
        if g[axis] != 0.0:
            ax = 2 - axis
            sl = [slice(None)] * 3
            sl[ax] = slice(1, -1)
            f[tuple(sl)] = f[tuple(sl)] + dt * g[axis]
        out.append(f)
    return tuple(out)


def zero_walls(u, v, w):
    out = []
    for axis, f in enumerate((u, v, w)):
        f = f.copy()
        ax = 2 - axis
        sl = [slice(None)] * 3
        sl[ax] = 0
        f[tuple(sl)] = 0.0
        sl[ax] = -1
        f[tuple(sl)] = 0.0
        out.append(f)
    return tuple(out)


def step(phi, u, v, w, dx, dt, P, p0=None, order=3):
    """One timestep of the corrected specification, order 3:
    level set TVD-RK3 (Shu-Osher) with the step's initial velocity; velocity
    Shu-Osher RK3 over SolveForRK stages (WENO5 self-advection, wall faces
    zeroed, gravity, semi-implicit viscosity, projection correcting u, v and
    w); reinitialisation as the reference's RK3 of reinitialisation blocks
    (EULERIAN_FLUID_SOLVER_3D.h:1081-1109).  P is a dict with rho_neg,
    rho_pos, mu_neg, mu_pos, gravity, eps, reinit_iterations, reinit_scaling,
    tol, max_iter, viscosity (bool, or "explicit" for the reference's air/water
    update, with viscosity_in_place for its in-place order), visc_tol.  Returns (phi, u, v, w, p, info)."""
    eps = P["eps"]
    L = lambda f: weno5_levelset(f, u, v, w, dx, dt, eps)
    phi1 = L(phi)
    if order == 3:
        phi2 = 0.75 * phi + 0.25 * L(phi1)
        phin = (1.0 / 3.0) * phi + (2.0 / 3.0) * L(phi2)
    else:  # Heun (EULERIAN_FLUID_SOLVER_3D.h:809-832, 888-911)
        phin = 0.5 * phi + 0.5 * L(phi1)
    p = np.zeros_like(phi) if p0 is None else p0
    info = {"iterations": [], "rel_residual": []}

    def stage(vel, c0, c1, base):
        nonlocal p
        a = eno3_velocity(*vel, dx, dt) if P.get("velocity_eno3", False) else weno5_velocity(*vel, dx, dt, eps)
        a = zero_walls(*a)
        a = add_gravity(*a, P["gravity"], dt)
        if P.get("viscosity", True) == "explicit":
            a = explicit_viscosity(phin, *a, dx, dt, P["rho_neg"], P["rho_pos"], P["mu_neg"], P["mu_pos"],
                                   faithful=P.get("viscosity_in_place", False))
        elif P.get("viscosity", True):
            a, _ = viscosity_semi_implicit(phin, *a, dx, dt, P["rho_neg"], P["rho_pos"], P["mu_neg"], P["mu_pos"],
                                           P["visc_tol"], 10000, "rel")
        uu, vv, ww, p, pi = projection(phin, *a, dx, dt, P["rho_neg"], P["rho_pos"], P["tol"], P["max_iter"],
                                       mode="corrected", criterion="rel", p0=p, sigma=P.get("sigma", 0.0),
                                       curvature_typo=P.get("curvature_typo", False))
        info["iterations"].append(pi["iterations"])
        info["rel_residual"].append(pi["rel_residual"])
        out = (uu, vv, ww)
        if c0 != 0.0:
            out = tuple(c0 * b + c1 * o for b, o in zip(base, out))
        return out

    base = (u, v, w)
    it, sc = P["reinit_iterations"], P["reinit_scaling"]
    sweep = [P.get("sweep_direction", 0)]

    def reinit(f):
        # EULERIAN_FLUID_SOLVER_3D::Reinitialization: fast sweeping (its
        # sweep_direction advancing per call), then the Sussman block
        if P.get("fast_sweeping", False):
            f = fast_sweeping(f, dx, sweep[0])
            sweep[0] += 1
        return reinitialization_block(f, dx, it, sc, eps) if it > 0 else f

    if order == 3:
        s1 = stage(base, 0.0, 1.0, base)
        s2 = stage(s1, 0.75, 0.25, base)
        s3 = stage(s2, 1.0 / 3.0, 2.0 / 3.0, base)
        r1 = reinit(phin)
        r2 = 0.75 * phin + 0.25 * reinit(r1)
        phi_out = (1.0 / 3.0) * phin + (2.0 / 3.0) * reinit(r2)
    else:
        s3 = stage(base, 0.0, 1.0, base)
        if order == 2:
            s3 = stage(s3, 0.5, 0.5, base)
        r1 = reinit(phin)
        phi_out = 0.5 * phin + 0.5 * reinit(r1)
    info["sweep_direction"] = sweep[0]
    return phi_out, s3[0], s3[1], s3[2], p, info


# ----------------------------------------------------------------------------
# Surface output: marching cubes (WRITE_LEVELSET.h:22-84,
# MARCHING_CUBES_ALGORITHM.h:146-166, 497-757, FIELD_STRUCTURE_3D.h:225-251)
# ----------------------------------------------------------------------------

# Cube corners: bit 0 the x offset, bit 1 y, bit 2 z from the cube's low
# corner.  Edges 0-3 run along x, 4-7 along y, 8-11 along z; faces list
# their corners in cyclic order.
MC_EDGES = ((0, 1), (2, 3), (4, 5), (6, 7), (0, 2), (1, 3), (4, 6), (5, 7), (0, 4), (1, 5), (2, 6), (3, 7))
MC_FACES = ((0, 2, 6, 4), (1, 3, 7, 5), (0, 1, 5, 4), (2, 3, 7, 6), (0, 1, 3, 2), (4, 5, 7, 6))


def marching_cubes_table():
    """For each of the 256 inside/outside patterns of a cube (bit c set when
    corner c has phi <= 0), the triangles as triples of cube edges.

    The surface crosses each face along segments between its sign-changing
    edges; a face whose diagonal corners share a sign (four crossings) cuts
    off each inside corner, a rule that both cubes of the face apply alike,
    so the mesh is closed.  The segments of the six faces close into loops,
    each loop is fanned from its lowest edge.  The reference's own table
    (MARCHING_CUBES_ALGORITHM_TABLE.h) gives the same crossings and the
    same loops on the unambiguous patterns; its triangles differ."""
    edge_of = {frozenset(e): k for k, e in enumerate(MC_EDGES)}
    table = []
    for mask in range(256):
        inside = [(mask >> c) & 1 for c in range(8)]
        partner = {}
        for f in MC_FACES:
            ring = [edge_of[frozenset((f[q], f[(q + 1) % 4]))] for q in range(4)]
            active = [inside[f[q]] != inside[f[(q + 1) % 4]] for q in range(4)]
            if sum(active) == 2:
                segs = [tuple(ring[q] for q in range(4) if active[q])]
            elif sum(active) == 4:
                segs = [(ring[(q - 1) % 4], ring[q]) for q in range(4) if inside[f[q]]]
            else:
                segs = []
            for a, b in segs:
                partner.setdefault(a, []).append(b)
                partner.setdefault(b, []).append(a)
        tris, seen = [], set()
        for start in sorted(partner):
            if start in seen:
                continue
            loop, prev, cur = [start], None, start
            seen.add(start)
            while True:
                a, b = partner[cur]
                nxt = b if a == prev else a
                if nxt == start:
                    break
                loop.append(nxt)
                seen.add(nxt)
                prev, cur = cur, nxt
            tris += [(loop[0], loop[q], loop[q + 1]) for q in range(1, len(loop) - 1)]
        table.append(tris)
    return table


def mc_node_coordinate(I, n, dx):
    """A cube corner's coordinate along one axis as the reference forms it
    (MARCHING_CUBES_ALGORITHM.h:151-166): the centre of cube i = min(I, n-1)
    from the domain's low end 0, then -+ half a cell."""
    half = dx * 0.5
    i = min(I, n - 1)
    centre = (0.0 + half) + dx * float(i)
    return centre - half if I < n else centre + half


def mc_node_values(phi, dx):
    """phi at the cube corners: FIELD_STRUCTURE_3D::TriLinearInterpolation
    (FIELD_STRUCTURE_3D.h:225-251) with its indices clamped to the cells
    (the reference reads copied ghosts there), and phi == 0 moved to -1e-8
    (MARCHING_CUBES_ALGORITHM.h:308).  Returns the values [nz+1, ny+1, nx+1]
    and the corner coordinates per axis."""
    nz, ny, nx = phi.shape
    inv = 1.0 / dx
    xs = [mc_node_coordinate(I, nx, dx) for I in range(nx + 1)]
    ys = [mc_node_coordinate(J, ny, dx) for J in range(ny + 1)]
    zs = [mc_node_coordinate(K, nz, dx) for K in range(nz + 1)]

    def axis(pos, n):
        i0 = math.floor((pos - 0.0) * inv - 0.5)
        a = (pos - (0.0 + (0.5 + float(i0)) * dx)) * inv
        return min(max(i0, 0), n - 1), min(max(i0 + 1, 0), n - 1), a

    ax = [axis(p, nx) for p in xs]
    ay = [axis(p, ny) for p in ys]
    az = [axis(p, nz) for p in zs]
    f = phi.tolist()
    out = np.empty((nz + 1, ny + 1, nx + 1))
    for K, (k0, k1, c) in enumerate(az):
        for J, (j0, j1, b) in enumerate(ay):
            mamb_rows = None
            for I, (i0, i1, a) in enumerate(ax):
                v000, v100, v010, v001 = f[k0][j0][i0], f[k0][j0][i1], f[k0][j1][i0], f[k1][j0][i0]
                v110, v101, v011, v111 = f[k0][j1][i1], f[k1][j0][i1], f[k1][j1][i0], f[k1][j1][i1]
                mamb = (1.0 - a) * (1.0 - b)
                bc = b * c
                val = (v000 * (mamb * (1.0 - c)) + (a * (1.0 - b) * (1.0 - c)) * v100 + ((1.0 - a) * b * (1.0 - c)) * v010
                       + (mamb * c) * v001 + (a * b * (1.0 - c)) * v110 + (a * (1.0 - b) * c) * v101
                       + ((1.0 - a) * bc) * v011 + (a * bc) * v111)
                out[K, J, I] = -1e-8 if val == 0.0 else val
    return out, (np.array(xs), np.array(ys), np.array(zs))


def marching_cubes(phi, dx, table=None):
    """The zero level set as a closed triangle mesh, the form
    WRITE_LEVELSET::WriteOBJ writes: cube corners sampled as in
    mc_node_values; cubes with a corner at 4 dx or more skipped
    (MARCHING_CUBES_ALGORITHM.h:310-316); one vertex per crossed edge used by
    a kept cube, at (|phi1| P0 + |phi0| P1) * (1/(|phi0| + |phi1|)) (the
    reference's expression, VECTOR_3D.h:130-135 dividing by a reciprocal);
    triangles from marching_cubes_table, each turned so its normal
    (v1 - v0) x (v2 - v0) has a non-negative dot product with the gradient
    of the cube's trilinear phi at its centre; vertex normals the
    normalised sum of the unit normals of their triangles
    (VERTEX::DetermineNormal, TRIANGULAR_SURFACE.cpp:99-121).

    Vertices are numbered by edge: all x edges, then y, then z edges, each
    set in (k, j, i) order; triangles by cube in (k, j, i) order.  Returns
    (vertices [nv, 3] as (x, y, z), normals [nv, 3], triangles [nt, 3] with
    1-based vertex numbers)."""
    if table is None:
        table = marching_cubes_table()
    nz, ny, nx = phi.shape
    node, (xs, ys, zs) = mc_node_values(phi, dx)
    big = 4.0 * dx
    kept = np.ones((nz, ny, nx), dtype=bool)
    for dk in (0, 1):
        for dj in (0, 1):
            for di in (0, 1):
                kept &= node[dk:nz + dk, dj:ny + dj, di:nx + di] < big
    neg = node <= 0.0
    # edges: x edges [nz+1, ny+1, nx], y [nz+1, ny, nx+1], z [nz, ny+1, nx+1]
    cross = [neg[:, :, 1:] != neg[:, :, :-1], neg[:, 1:, :] != neg[:, :-1, :], neg[1:, :, :] != neg[:-1, :, :]]
    usedc = [np.zeros_like(c) for c in cross]
    for dk in (0, 1):
        for dj in (0, 1):
            # cubes touching x edge (k, j, i): cube (k-dk, j-dj, i)
            u = usedc[0]
            sub = np.zeros_like(u)
            sub[dk:dk + nz, dj:dj + ny, :] |= kept
            u |= sub
            sub = np.zeros_like(usedc[1])
            sub[dk:dk + nz, :, dj:dj + nx] |= kept
            usedc[1] |= sub
            sub = np.zeros_like(usedc[2])
            sub[:, dk:dk + ny, dj:dj + nx] |= kept
            usedc[2] |= sub
    used = [c & u for c, u in zip(cross, usedc)]
    ids, verts, base = [], [], 0
    for axis, u in enumerate(used):
        idx = np.full(u.shape, -1, dtype=np.int64)
        n = int(u.sum())
        idx[u] = base + np.arange(n)
        ids.append(idx)
        for (k, j, i) in zip(*np.nonzero(u)):
            k0, j0, i0 = k, j, i
            k1, j1, i1 = k + (axis == 2), j + (axis == 1), i + (axis == 0)
            p0, p1 = node[k0, j0, i0], node[k1, j1, i1]
            a0, a1 = (p0 if p0 > 0 else -p0), (p1 if p1 > 0 else -p1)
            inv = 1.0 / (a0 + a1)
            P0 = (xs[i0], ys[j0], zs[k0])
            P1 = (xs[i1], ys[j1], zs[k1])
            verts.append([(a1 * P0[q] + a0 * P1[q]) * inv for q in range(3)])
        base += n
    verts = np.array(verts, dtype=float).reshape(-1, 3)

    def edge_vertex(e, k, j, i):
        c0, c1 = MC_EDGES[e]
        kk, jj, ii = k + (c0 >> 2 & 1), j + (c0 >> 1 & 1), i + (c0 & 1)
        return int(ids[0 if e < 4 else (1 if e < 8 else 2)][kk, jj, ii])

    tris = []
    for (k, j, i) in zip(*np.nonzero(kept)):
        c = [node[k + (q >> 2 & 1), j + (q >> 1 & 1), i + (q & 1)] for q in range(8)]
        mask = sum(1 << q for q in range(8) if c[q] <= 0.0)
        if not table[mask]:
            continue
        g = np.array([((c[1] + c[3]) + (c[5] + c[7])) - ((c[0] + c[2]) + (c[4] + c[6])),
                      ((c[2] + c[3]) + (c[6] + c[7])) - ((c[0] + c[1]) + (c[4] + c[5])),
                      ((c[4] + c[5]) + (c[6] + c[7])) - ((c[0] + c[1]) + (c[2] + c[3]))])
        for (e0, e1, e2) in table[mask]:
            v0, v1, v2 = edge_vertex(e0, k, j, i), edge_vertex(e1, k, j, i), edge_vertex(e2, k, j, i)
            P0, P1, P2 = verts[v0], verts[v1], verts[v2]
            nrm = np.cross(P1 - P0, P2 - P0)
            if nrm[0] * g[0] + nrm[1] * g[1] + nrm[2] * g[2] < 0.0:
                v1, v2 = v2, v1
            tris.append((v0, v1, v2))
    tris = np.array(tris, dtype=np.int64).reshape(-1, 3)
    normals = np.zeros_like(verts)
    if len(tris):
        P = verts[tris]
        fn = np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0])
        ln = np.linalg.norm(fn, axis=1)
        fn = np.where(ln[:, None] > 0, fn / np.where(ln > 0, ln, 1.0)[:, None], 0.0)
        for q in range(3):
            np.add.at(normals, tris[:, q], fn)
        ln = np.linalg.norm(normals, axis=1)
        normals = np.where(ln[:, None] > 0, normals / np.where(ln > 0, ln, 1.0)[:, None], 0.0)
    return verts, normals, tris + 1


# ----------------------------------------------------------------------------
# Oil/water pipe mode, vertical pipe (axis y): the level-set path and the
# dimensionless forcing (ADVECTION_3D.h:204-242, 360-378, 380-430;
# ADVECTION_METHOD_3D.h:281-523; FIELD_STRUCTURE_3D.h:1328-1431;
# EULERIAN_FLUID_SOLVER_3D.h:496-514, 2198-2225, 2237-2330)
# ----------------------------------------------------------------------------

def pipe_grids(n, lo, hi):
    """The reference's cell grid and the three MAC face grids
    (GRID_STRUCTURE_3D.h:91-137, EULERIAN_FLUID_SOLVER_3D.h:405-427): per
    grid (x_min, y_min, z_min, dx, dy, dz).  Positions are x_min + i*dx (the
    reference's node convention), each face grid spans half a cell beyond the
    cell grid on its own axis, and every spacing is (max - min)/(res - 1)."""
    nx, ny, nz = n
    (x0, y0, z0), (x1, y1, z1) = lo, hi
    d = ((x1 - x0) / (nx - 1), (y1 - y0) / (ny - 1), (z1 - z0) / (nz - 1))
    cells = (x0, y0, z0) + d
    grids = [cells]
    res = (nx, ny, nz)
    for axis in range(3):
        mn, mx, r = [x0, y0, z0], [x1, y1, z1], list(res)
        mn[axis] = mn[axis] - 0.5 * d[axis]
        mx[axis] = mx[axis] + 0.5 * d[axis]
        r[axis] += 1
        grids.append(tuple(mn) + tuple((mx[q] - mn[q]) / (r[q] - 1) for q in range(3)))
    return grids


def pipe_constants(a, R2, m, eta, K, g, water_density, oil_density, water_viscosity, oil_viscosity,
                   surface_tension):
    """The dimensionless constants of the core-annular pipe flow the reference
    derives from its script (EULERIAN_FLUID_SOLVER_3D.h:496-514)."""
    R1 = R2 / a
    f = 1.0 / (K - 1.0) * g * (oil_density - K * water_density)
    A = (a * a - 1.0) + (m * K + 2.0 * (K - 1) * math.log(a))
    V0 = (f + water_density * g) * (R1 * R1) / (4.0 * water_viscosity) * A
    J = surface_tension * R1 * oil_density / (oil_viscosity * oil_viscosity)
    Re = (oil_density * R1 * abs(V0)) / oil_viscosity
    We = (1.0 / J) * (Re * Re)
    return dict(a=a, R1=R1, m=m, eta=eta, K=K, g=g, f=f, A=A, V0=V0, J=J, Re=Re, We=We)


def pipe_boundary(grid, shape, a):
    """Distance to the pipe wall, sqrt(x^2 + z^2) - a, at the points of one
    grid (vertical pipe; EULERIAN_FLUID_SOLVER_3D.h:2282-2300)."""
    x0, _, z0, dx, _, dz = grid
    nz, ny, nx = shape
    x = x0 + np.arange(nx) * dx
    z = z0 + np.arange(nz) * dz
    r = np.sqrt(x[None, :] * x[None, :] + z[:, None] * z[:, None]) - a
    return np.broadcast_to(r[:, None, :], shape).copy()


def periodic_ghosts_y(phi, g=G):
    """Ghosted copy of a cell field, periodic along y with the reference's
    node convention (FIELD_STRUCTURE_3D.h:1328-1431): the first and last
    cells are the same point, so ghost j0 - m is cell j1 - m and ghost j1 + m
    is cell j0 + m.  Only the y ghosts of interior columns are written: the x
    and z ghost layers of the reference's ghost copy are never filled in a
    vertical pipe and hold zero."""
    nz, ny, nx = phi.shape
    a = np.zeros((nz + 2 * g, ny + 2 * g, nx + 2 * g))
    a[g:g + nz, g:g + ny, g:g + nx] = phi
    for m in range(1, g + 1):
        a[g:g + nz, g - m, g:g + nx] = phi[:, ny - 1 - m, :]
        a[g:g + nz, g + ny - 1 + m, g:g + nx] = phi[:, m, :]
    return a


def _wall_extrapolate(vel_ghost, b, along):
    """Velocity ghost values on faces outside the pipe next to faces inside
    it (ADVECTION_3D.h:445-485): zero where all four transverse neighbours are
    outside, else (theta-1)/theta times the inside neighbour along `along`
    (numpy axis), theta = |b_in|/(|b_in| + |b_out|); the + side wins when both
    sides are inside.  b outside the face grid counts as 0 (neither side)."""
    out = vel_ghost.copy()
    bp = np.pad(b, 1)  # the unfilled ghost layer of the boundary array holds 0
    c = (slice(1, -1),) * 3

    def nb(ax, s):
        sl = list(c)
        sl[ax] = slice(1 + s, bp.shape[ax] - 1 + s)
        return bp[tuple(sl)]

    vp = np.pad(vel_ghost, 1)

    def vnb(ax, s):
        sl = list(c)
        sl[ax] = slice(1 + s, vp.shape[ax] - 1 + s)
        return vp[tuple(sl)]

    outside = b > 0
    all4 = (nb(2, -1) > 0) & (nb(2, 1) > 0) & (nb(0, -1) > 0) & (nb(0, 1) > 0)
    out = np.where(outside & all4, 0.0, out)
    for s in (-1, 1):
        bn = nb(along, s)
        with np.errstate(divide="ignore", invalid="ignore"):
            theta = np.abs(bn) / (np.abs(bn) + np.abs(b))
            ext = (theta - 1) / theta * vnb(along, s)
        out = np.where(outside & (bn < 0), ext, out)
    return out


def pipe_levelset_velocities(u, v, w, grids, a):
    """SetupBoundaryConditionForVelocity for the level-set advection of a
    vertical pipe (ADVECTION_3D.h:380-490): the face velocities outside the
    pipe become 0 in u and w (v is left alone); the ghost copies the WENO5
    update reads hold the velocities inside the pipe (FIELD_STRUCTURE_3D.h:
    1432-1460, 0 outside) and, on x and z faces just outside it, the
    extrapolation across the wall.  Returns (u, v, w, ug, vg, wg)."""
    bx = pipe_boundary(grids[1], u.shape, a)
    by = pipe_boundary(grids[2], v.shape, a)
    bz = pipe_boundary(grids[3], w.shape, a)
    ug = np.where(bx < 1e-8, u, 0.0)
    vg = np.where(by < 1e-8, v, 0.0)
    wg = np.where(bz < 1e-8, w, 0.0)
    # the y component's periodic fill also rewrites its first and last face
    # rows (face 0 is face ny-1, face ny is face 1: FIELD_STRUCTURE_3D.h:
    # 1466-1500), where the face is inside
    ny = v.shape[1] - 1
    vg[:, 0, :] = np.where(by[:, 0, :] < 1e-8, v[:, ny - 1, :], vg[:, 0, :])
    vg[:, ny, :] = np.where(by[:, ny, :] < 1e-8, v[:, 1, :], vg[:, ny, :])
    ug = _wall_extrapolate(ug, bx, 2)
    wg = _wall_extrapolate(wg, bz, 0)
    return np.where(bx > 0, 0.0, u), v.copy(), np.where(bz > 0, 0.0, w), ug, vg, wg


def pipe_weno5_levelset(phi, u, v, w, grids, a, dt, eps):
    """ADVECTION_3D::Solve_Levelset of a vertical pipe: the velocity set-up
    above, then WENO5th with the boundary level set (ADVECTION_METHOD_3D.h:
    281-523): cells outside the pipe keep their value, the rest take the
    WENO5 upwind update on the periodic ghost copy, with the per-axis
    spacings of the cell grid.  Returns (phi, u, v, w)."""
    u2, v2, w2, ug, vg, wg = pipe_levelset_velocities(u, v, w, grids, a)
    cg = grids[0]
    pg = periodic_ghosts_y(phi)
    dxm, dxp = weno5_derivatives(pg, 0, 1.0 / cg[3], eps)
    dym, dyp = weno5_derivatives(pg, 1, 1.0 / cg[4], eps)
    dzm, dzp = weno5_derivatives(pg, 2, 1.0 / cg[5], eps)
    uc = (ug[:, :, 1:] + ug[:, :, :-1]) * 0.5
    vc = (vg[:, 1:, :] + vg[:, :-1, :]) * 0.5
    wc = (wg[1:, :, :] + wg[:-1, :, :]) * 0.5
    new = _upwind_update(phi, dt, uc, vc, wc, dxm, dxp, dym, dyp, dzm, dzp)
    bl = pipe_boundary(cg, phi.shape, a)
    return np.where(bl > 0, phi, new), u2, v2, w2


def pipe_reinitialization(phi, grids, iterations, scaling, eps, typo=True):
    """EULERIAN_FLUID_SOLVER_3D::Reinitialization of a pipe: S from the
    block's input, then `iterations` Sussman pseudo-steps of dx/scaling, each
    reading the periodic ghost copy (ADVECTION_3D.h:360-378).  The reference
    runs its tree with the two typo leaves (typo=True)."""
    dx = grids[0][3]
    s = sign_function(phi, dx)
    dtau = dx / scaling
    for _ in range(iterations):
        phi = sussman_step(phi, s, dx, dtau, eps, typo, ghost_source=periodic_ghosts_y(phi))
    return phi


def pipe_forcing(phi, v, grids, C, gravity_y, oil_density, dt, fixed_v=None):
    """The dimensionless body force of a vertical pipe (ApplyGravity,
    EULERIAN_FLUID_SOLVER_3D.h:2304-2326): on y faces inside the pipe that are
    not fixed, v += R1/V0^2 (dt g_y + dt f/(rho_oil rho_f)), rho_f = 1 +
    (eta - 1) H(phi_f) the smeared density of the face's level set
    phi_f = (phi_c + phi_below)/2 from the periodic ghost copy, H with
    epsilon = 1.5 dy."""
    cg, vgrid = grids[0], grids[2]
    pg = periodic_ghosts_y(phi)
    nz, ny, nx = phi.shape
    col = pg[G:G + nz, :, G:G + nx]
    phi_f = 0.5 * (col[:, G:G + ny + 1, :] + col[:, G - 1:G + ny, :])
    h = heaviside_projection(phi_f, 1.5 * cg[4])
    rho_f = 1.0 + (C["eta"] - 1.0) * h
    by = pipe_boundary(vgrid, v.shape, C["a"])
    add = C["R1"] / (C["V0"] * C["V0"]) * (dt * gravity_y + 1.0 / (oil_density * rho_f) * (dt * C["f"]))
    mask = by < 0
    if fixed_v is not None:
        mask &= ~fixed_v
    return np.where(mask, v + add, v)


def _pipe_periodic_copy(c, b, y_component):
    """The masked periodic ghost copy of one face component of a vertical pipe
    (FIELD_STRUCTURE_3D.h:1432-1540): interior = c where b < 1e-8, else 0;
    the y ghost rows of interior columns hold the periodic images of c (the
    reference tests b there on its unfilled ghost rows, which hold 0); for the
    y component the first and last face rows are rewritten with their images
    where b < 1e-8 too (face 0 is face ny-1, face ny is face 1).  Faces outside
    the pipe in a row or column that crosses it take the linear extrapolation
    below; the rest of the x and z ghost layers hold 0."""
    g = G
    nz, Ny, nx = c.shape
    out = np.zeros((nz + 2 * g, Ny + 2 * g, nx + 2 * g))
    inner = np.where(b < 1e-8, c, 0.0)
    if y_component:
        inner[:, 0, :] = np.where(b[:, 0, :] < 1e-8, c[:, Ny - 2, :], inner[:, 0, :])
        inner[:, Ny - 1, :] = np.where(b[:, Ny - 1, :] < 1e-8, c[:, 1, :], inner[:, Ny - 1, :])
        lo = lambda m: c[:, Ny - 2 - m, :]
        hi = lambda m: c[:, 1 + m, :]
    else:
        lo = lambda m: c[:, Ny - 1 - m, :]
        hi = lambda m: c[:, m, :]
    out[g:g + nz, g:g + Ny, g:g + nx] = inner
    for m in range(1, g + 1):
        out[g:g + nz, g - m, g:g + nx] = lo(m)
        out[g:g + nz, g + Ny - 1 + m, g:g + nx] = hi(m)
    # then, along each row and column of the pipe's cross-section, every face
    # from the first one outside the pipe to the end of the row (ghost layers
    # included) takes the linear extrapolation of the velocity itself,
    # 2 c(t-1) - c(t-2) outward (FIELD_STRUCTURE_3D.h:1563-1610): x rows
    # first, right then left side, then z columns, which overwrite
    cp = np.pad(c, g)  # the velocity's own ghost layers hold 0
    bp = np.pad(b, 1)  # the boundary array's unfilled ghost layer holds 0
    for (k, j, i) in np.argwhere((bp[1:-1, 1:-1, :-2] < 0) & (b > 0)):  # x: inside at i-1
        for t in range(i, nx + g):
            out[k + g, j + g, t + g] = 2.0 * cp[k + g, j + g, t - 1 + g] - cp[k + g, j + g, t - 2 + g]
    for (k, j, i) in np.argwhere((bp[1:-1, 1:-1, 2:] < 0) & (b > 0)):  # x: inside at i+1
        for t in range(i, -g - 1, -1):
            out[k + g, j + g, t + g] = 2.0 * cp[k + g, j + g, t + 1 + g] - cp[k + g, j + g, t + 2 + g]
    for (k, j, i) in np.argwhere((bp[:-2, 1:-1, 1:-1] < 0) & (b > 0)):  # z: inside at k-1
        for t in range(k, nz + g):
            out[t + g, j + g, i + g] = 2.0 * cp[t - 1 + g, j + g, i + g] - cp[t - 2 + g, j + g, i + g]
    for (k, j, i) in np.argwhere((bp[2:, 1:-1, 1:-1] < 0) & (b > 0)):  # z: inside at k+1
        for t in range(k, -g - 1, -1):
            out[t + g, j + g, i + g] = 2.0 * cp[t + 1 + g, j + g, i + g] - cp[t + 2 + g, j + g, i + g]
    return out


def _pipe_eno_guard(gc, b, axis):
    """The copy of a component that the pipe's ENO3 reads along x (axis 0) or
    z (axis 2) (ADVECTION_3D.h:560-700): next to each inside face whose
    neighbour along the axis is outside, the neighbour gets the value
    extrapolated across the wall, (theta-1)/theta times the inside face's,
    theta = |b_in|/(|b_in| + |b_out|), and the next three faces the large
    values (10t)^t, t = 2, 3, 4, so that the ENO stencil choice stays inside
    the pipe."""
    g = G
    out = gc.copy()
    ax = 2 - axis
    nz, Ny, nx = b.shape
    for s in (1, -1):
        bn = np.zeros_like(b)
        src = [slice(None)] * 3
        dst = [slice(None)] * 3
        if s == 1:
            src[ax], dst[ax] = slice(1, None), slice(0, -1)
        else:
            src[ax], dst[ax] = slice(0, -1), slice(1, None)
        bn[tuple(dst)] = b[tuple(src)]
        idx = np.argwhere((b < 0) & (bn > 0))
        for (k, j, i) in idx:
            pos = [k + g, j + g, i + g]
            theta = abs(b[k, j, i]) / (abs(bn[k, j, i]) + abs(b[k, j, i]))
            p1 = list(pos)
            p1[ax] += s
            out[tuple(p1)] = (theta - 1) / theta * gc[tuple(pos)]
            for t in range(2, 5):
                pt = list(pos)
                pt[ax] += s * t
                out[tuple(pt)] = float((10 * t) ** t)
    return out


def pipe_fixed_faces(n):
    """The centre-line faces Solve_Velocity holds fixed in a vertical pipe
    (ADVECTION_3D.h:246-275): x faces i = nx/2, nx/2 + 1 and z faces k =
    nz/2, nz/2 + 1 at the centre of the other axis, the y faces of the centre
    column (integer halves of the face grids' last indices)."""
    nx, ny, nz = n
    fu = np.zeros((nz, ny, nx + 1), bool)
    fv = np.zeros((nz, ny + 1, nx), bool)
    fw = np.zeros((nz + 1, ny, nx), bool)
    fu[(nz - 1) // 2, :, nx // 2] = True
    fu[(nz - 1) // 2, :, nx // 2 + 1] = True
    fv[(nz - 1) // 2, :, (nx - 1) // 2] = True
    fw[nz // 2, :, (nx - 1) // 2] = True
    fw[nz // 2 + 1, :, (nx - 1) // 2] = True
    return fu, fv, fw


def pipe_eno3_velocity(u, v, w, grids, a, dt):
    """ADVECTION_3D::Solve_Velocity of a vertical pipe with ENO3
    (ADVECTION_3D.h:244-358, ADVECTION_METHOD_3D.h:1935-2240): each face
    inside the pipe and not fixed takes the ENO3 upwind update, its x and z
    derivatives from the guarded copies, its y derivative and the advecting
    velocities from the masked periodic copies; the other faces keep their
    value.  Returns (u, v, w)."""
    comps = (u, v, w)
    bs = [pipe_boundary(grids[1 + ax], comps[ax].shape, a) for ax in range(3)]
    gen = [_pipe_periodic_copy(comps[ax], bs[ax], ax == 1) for ax in range(3)]
    nz, ny, nx = u.shape[0], u.shape[1], u.shape[2] - 1
    fixed = pipe_fixed_faces((nx, ny, nz))
    out = []
    for ax in range(3):
        gx = _pipe_eno_guard(gen[ax], bs[ax], 0)
        gz = _pipe_eno_guard(gen[ax], bs[ax], 2)
        gr = grids[1 + ax]
        uvel, vvel, wvel = _face_velocities(ax, gen[0], gen[1], gen[2])
        dxm, dxp = eno3_derivatives(gx, 0, gr[3])
        dym, dyp = eno3_derivatives(gen[ax], 1, gr[4])
        dzm, dzp = eno3_derivatives(gz, 2, gr[5])
        new = _upwind_update(comps[ax], dt, uvel, vvel, wvel, dxm, dxp, dym, dyp, dzm, dzp)
        out.append(np.where((bs[ax] < 0) & ~fixed[ax], new, comps[ax]))
    return tuple(out)


# ----------------------------------------------------------------------------
# Oil/water pipe mode, vertical pipe: the projection (PROJECTION_3D.h:416-441,
# 596-834, 849-1097, 1099-1449, 1475-1610; POISSON_SOLVER_3D.h:165-252,
# 527-552, 1360-1819)
# ----------------------------------------------------------------------------

def pipe_fluid_cells(grids, shape, a):
    """The cells that are unknowns of the pipe's pressure system: wall distance
    <= 0 (SetupBoundaryConditions, Neumann + cylindrical_boundary + is_vertical,
    PROJECTION_3D.h:1017-1040, marks the others BC_NEUM)."""
    return pipe_boundary(grids[0], shape, a) <= 0


def pipe_density(phi, water_density, oil_density):
    """DetermineProjectionDensity in the dimensionless form (PROJECTION_3D.h:
    642-669): 1 in the oil (phi <= 0), water_density/oil_density in the water."""
    return np.where(phi <= 0, 1.0, water_density / oil_density)


def pipe_divergence(u, v, w, grids, a, dt):
    """DetermineDivergence of the pipe (PROJECTION_3D.h:697-719, 1519-1610):
    the MAC divergence of the masked periodic velocity copies with the linear
    wall extrapolation on x and z faces just outside the pipe (the copies the
    level-set advection reads; the projection's if/else chain prefers the -
    side where the advection's prefers the +, which differ only on faces
    outside the pipe with an inside neighbour on both sides, impossible for a
    convex wall), zero in cells outside the pipe, then scaled by 1/dt."""
    _, _, _, ug, vg, wg = pipe_levelset_velocities(u, v, w, grids, a)
    cg = grids[0]
    d = (1.0 / cg[3]) * (ug[:, :, 1:] - ug[:, :, :-1])
    d = d + (1.0 / cg[4]) * (vg[:, 1:, :] - vg[:, :-1, :])
    d = d + (1.0 / cg[5]) * (wg[1:, :, :] - wg[:-1, :, :])
    d = np.where(pipe_boundary(cg, d.shape, a) > 0, 0.0, d)
    return d * (1.0 / dt)


def _periodic_y_pad1(f):
    """One ghost layer around a cell field: the y ghosts of interior columns
    are the periodic images (node convention: ghost -1 is cell ny-2, ghost ny
    is cell 1; FIELD_STRUCTURE_3D.h:1328-1431), the x and z ghost layers 0."""
    nz, ny, nx = f.shape
    out = np.zeros((nz + 2, ny + 2, nx + 2))
    out[1:-1, 1:-1, 1:-1] = f
    out[1:-1, 0, 1:-1] = f[:, ny - 2, :]
    out[1:-1, ny + 1, 1:-1] = f[:, 1, :]
    return out


def pipe_poisson(phi, fluid, var, dx, deflate=True):
    """The pipe's pressure matrix (oil/water branch of
    BuildLinearSystemNodeJumpConditionVaribleCoefficient, POISSON_SOLVER_3D.h:
    1360-1499) in the matrix-free form of poisson_operator: couplings
    beta/dx^2 only between two unknowns (cells of the pipe), the diagonal the
    sum of those betas in the order l, r, b, t, d, u; the first unknown in
    the reference's row order (k, j, i) adds the beta of its down neighbour,
    a Neumann cell below the pipe's lowest row, computed from that cell's
    level set and 1/rho (the deflation; its other Neumann arms add 0); a
    zero sum becomes 1.  Cells outside the pipe get diagonal 1 and no
    coupling (they are not unknowns)."""
    nz, ny, nx = phi.shape
    ab = np.abs(phi)

    def beta(vc, vn, ac, an):
        with np.errstate(invalid="ignore", divide="ignore"):
            return vc * vn * (an + ac) / (vn * ac + vc * an)

    bx = np.zeros((nz, ny, nx + 1)); by = np.zeros((nz, ny + 1, nx)); bz = np.zeros((nz + 1, ny, nx))
    bx[:, :, 1:-1] = np.where(fluid[:, :, :-1] & fluid[:, :, 1:],
                              beta(var[:, :, :-1], var[:, :, 1:], ab[:, :, :-1], ab[:, :, 1:]), 0.0)
    by[:, 1:-1, :] = np.where(fluid[:, :-1, :] & fluid[:, 1:, :],
                              beta(var[:, :-1, :], var[:, 1:, :], ab[:, :-1, :], ab[:, 1:, :]), 0.0)
    bz[1:-1, :, :] = np.where(fluid[:-1, :, :] & fluid[1:, :, :],
                              beta(var[:-1, :, :], var[1:, :, :], ab[:-1, :, :], ab[1:, :, :]), 0.0)
    inv2 = 1.0 / (dx * dx)
    coef = ((((bx[:, :, :-1] + bx[:, :, 1:]) + by[:, :-1, :]) + by[:, 1:, :]) + bz[:-1, :, :]) + bz[1:, :, :]
    first = tuple(int(q) for q in np.argwhere(fluid)[0])  # (k, j, i) of row 0
    if deflate:
        k, j, i = first
        vc, vd, ac, ad = var[k, j, i], var[k - 1, j, i], ab[k, j, i], ab[k - 1, j, i]
        coef[k, j, i] = coef[k, j, i] + vc * vd * (ad + ac) / (vc * ad + vd * ac)
    coef = np.where(fluid & (coef == 0), 1.0, coef)
    coef = np.where(fluid, coef, 1.0 / inv2)
    return bx * inv2, by * inv2, bz * inv2, inv2 * coef, first


def pipe_jump_terms(phi, jc, var, dx):
    """The jump terms F_X, F_Y, F_Z of the pipe's right-hand side
    (POISSON_SOLVER_3D.h:1690-1788, jc_on_derivative = 0), every arm of an
    unknown included: arms into Neumann cells too.  The y arms of the first
    and last rows read the level set's clamped ghost (ComputeNormals,
    LEVELSET_3D.h:931, fills the ghosts by copying the nearest cell just
    before the system is built), so they never cross the interface; jc and
    1/rho carry their periodic images there (PROJECTION_3D.h:778-827)."""
    pg = np.pad(phi, 1, mode="edge")
    vg = _periodic_y_pad1(var)
    jg = _periodic_y_pad1(jc)
    nz, ny, nx = phi.shape
    inv2 = 1.0 / (dx * dx)

    def nb(arr, di, dj, dk):
        return arr[1 + dk:1 + dk + nz, 1 + dj:1 + dj + ny, 1 + di:1 + di + nx]

    pc, vc, jcc = phi, var, jc
    ac = np.abs(pc)
    out = []
    for (lo, hi) in (((-1, 0, 0), (1, 0, 0)), ((0, -1, 0), (0, 1, 0)), ((0, 0, -1), (0, 0, 1))):
        F = []
        for d, low in ((lo, True), (hi, False)):
            pn, vn, jn = nb(pg, *d), nb(vg, *d), nb(jg, *d)
            an = np.abs(pn)
            with np.errstate(divide="ignore", invalid="ignore"):
                a = (jcc * an + jn * ac) / (ac + an)
                if low:
                    beta = vc * vn * (an + ac) / (vc * an + vn * ac)
                else:
                    beta = vc * vn * (an + ac) / (vn * ac + vc * an)
            f = np.where((pc <= 0) & (pn > 0), inv2 * a * beta,
                         np.where((pc > 0) & (pn <= 0), -inv2 * a * beta, 0.0))
            F.append(f)
        out.append(F[0] + F[1])
    return tuple(out)


def pipe_velocity_update(u, v, w, p, phi, jc, fluid, first, grids, dt, water_density, oil_density, fixed=None):
    """UpdateVelocityByPressureGradientVariableDensity of a vertical pipe
    (PROJECTION_3D.h:1099-1449).  A face whose + side cell is an unknown is
    updated when its - side cell is one too, or when the + side cell is the
    first unknown (row index 0 makes bc*bc_nb >= 0 hold against a Neumann
    cell, whose pressure stays 0); y faces only for 0 < j < ny.  Same-phase
    faces: -= dt (p_c - p_n)/rho_c/dx with the sharp density of the + side
    cell; faces crossing the interface: -= dt (p_c - p_n +- gamma)/rho_f/dx,
    gamma = (jc_c|phi_n| + jc_n|phi_c|)/(|phi_n| + |phi_c|), rho_f = 1 +
    (water/oil - 1) H(phi_f) with phi_f the face average from the periodic
    ghost copy and H of epsilon 1.5 dx.  Fixed faces keep their value.  Then
    the periodic copies: u and w row ny-1 = row 0; v row ny = row 1 and row
    0 = row ny-1."""
    cg = grids[0]
    h = (cg[3], cg[4], cg[5])
    nz, ny, nx = phi.shape
    rho_c = pipe_density(phi, water_density, oil_density)
    pgy = periodic_ghosts_y(phi)[G:G + nz, :, G:G + nx]  # periodic y ghosts, interior columns
    ratio = water_density / oil_density
    row0 = np.zeros_like(fluid)
    row0[first] = True
    out = [u.copy(), v.copy(), w.copy()]
    fixed = fixed if fixed is not None else (None, None, None)
    for axis in range(3):
        ax = 2 - axis
        sl_c = [slice(None)] * 3; sl_n = [slice(None)] * 3
        sl_c[ax] = slice(1, None); sl_n[ax] = slice(0, -1)
        sl_c, sl_n = tuple(sl_c), tuple(sl_n)
        ph_c, ph_n = phi[sl_c], phi[sl_n]
        if axis == 1:
            face_phi = 0.5 * (pgy[:, G + 1:G + ny, :] + pgy[:, G:G + ny - 1, :])
        else:
            face_phi = 0.5 * (ph_c + ph_n)
        rho_f = 1.0 + (ratio - 1.0) * heaviside_projection(face_phi, 1.5 * h[axis])
        with np.errstate(invalid="ignore", divide="ignore"):
            gamma = (jc[sl_c] * np.abs(ph_n) + jc[sl_n] * np.abs(ph_c)) / (np.abs(ph_n) + np.abs(ph_c))
        dp = p[sl_c] - p[sl_n]
        same = ph_c * ph_n > 0
        inv_h = 1.0 / h[axis]
        upd = np.where(same, dt * dp * (1.0 / rho_c[sl_c]) * inv_h,
                       np.where(ph_c <= 0, dt * (dp + gamma) * (1.0 / rho_f) * inv_h,
                                dt * (dp - gamma) * (1.0 / rho_f) * inv_h))
        ok = fluid[sl_c] & (fluid[sl_n] | row0[sl_c])
        fs = [slice(None)] * 3
        fs[ax] = slice(1, -1)
        fs = tuple(fs)
        if fixed[axis] is not None:
            ok = ok & ~fixed[axis][fs]
        f = out[axis]
        f[fs] = np.where(ok, f[fs] - upd, f[fs])
    out[0][:, ny - 1, :] = out[0][:, 0, :]
    out[1][:, ny, :] = out[1][:, 1, :]
    out[1][:, 0, :] = out[1][:, ny - 1, :]
    out[2][:, ny - 1, :] = out[2][:, 0, :]
    return tuple(out)


def pipe_projection(phi, u, v, w, grids, C, dt, tol, max_iter, water_density, oil_density, fixed=None, p0=None,
                    mode="faithful", criterion="abs"):
    """PROJECTION_3D::Solve of a vertical pipe with Neumann walls
    (cylindrical_boundary, dimensionless_form): divergence of the pipe's
    velocity copies, jump condition jc = kappa/We (PROJECTION_3D.h:758-768),
    the pipe's matrix (faithful: with the reference's deflation; corrected:
    the singular consistent system), right-hand side -div - F minus its mean
    over the unknowns (POISSON_SOLVER_3D.h:225-246), Jacobi-PCG from the
    previous pressure on the unknowns, and the pipe's velocity update.  The
    pressure of cells outside the pipe is not touched.  Returns
    (u, v, w, p, info)."""
    cg = grids[0]
    dx = cg[3]
    fluid = pipe_fluid_cells(grids, phi.shape, C["a"])
    rho = pipe_density(phi, water_density, oil_density)
    var = 1.0 / rho
    div = pipe_divergence(u, v, w, grids, C["a"], dt)
    kappa, _ = curvature(phi, dx, typo=True)
    jc = (1.0 / C["We"]) * kappa
    ax_, ay_, az_, diag, first = pipe_poisson(phi, fluid, var, dx, deflate=(mode == "faithful"))
    op = (ax_, ay_, az_, diag)
    FX, FY, FZ = pipe_jump_terms(phi, jc, var, dx)
    b = np.where(fluid, ((-div - FX) - FY) - FZ, 0.0)
    nrow = int(fluid.sum())
    b = np.where(fluid, b - (1.0 / nrow) * _seqsum(b[fluid]), 0.0)
    p_prev = np.zeros_like(phi) if p0 is None else p0
    x0 = np.where(fluid, p_prev, 0.0)
    x, it, rz, rel = pcg(lambda q: apply_poisson(op, q), diag, b, x0, tol, max_iter, criterion)
    p = np.where(fluid, x, p_prev)
    u2, v2, w2 = pipe_velocity_update(u, v, w, p, phi, jc, fluid, first, grids, dt, water_density, oil_density,
                                      fixed)
    return u2, v2, w2, p, {"iterations": it, "rz": rz, "rel_residual": rel, "b": b, "div": div, "jc": jc,
                           "fluid": fluid, "op": op}


def pipe_cfl_dt(u, v, w, grids, C, gravity_y, water_density, oil_density, kappa_max):
    """EULERIAN_FLUID_SOLVER_3D::CFLOneTimeStep in the pipe's dimensionless
    form with the semi-implicit viscosity (EULERIAN_FLUID_SOLVER_3D.h:
    2673-2785): 1/cfl, cfl = 0.5 (c + sqrt(c^2 + 4 g^2 + 4 s^2)) with
      c = max|u|/dx_u + max|v|/dy_v + max|w|/dz_w    (the face grids' spacings)
      g = sqrt(R1/V0^2 (|g_y| + |f/min(oil, water)|)/dy_v)
      s = sqrt((kappa_max/We)/(min(water/oil, 1) min(dx_u, dy_v, dz_w)^2))
    and no viscous term; kappa_max is max |kappa| over cells with
    |phi| < 0.1 of the last curvature the projection computed."""
    inv_x, inv_y, inv_z = 1.0 / grids[1][3], 1.0 / grids[2][4], 1.0 / grids[3][5]
    c_f = (float(np.max(np.abs(u))) * inv_x + float(np.max(np.abs(v))) * inv_y) + float(np.max(np.abs(w))) * inv_z
    g_f = math.sqrt(C["R1"] / (C["V0"] * C["V0"]) * (abs(gravity_y) + abs(1.0 / min(oil_density, water_density) * C["f"]))
                    * inv_y)
    h = min(grids[1][3], grids[2][4], grids[3][5])
    s_f = math.sqrt(((1.0 / C["We"]) * kappa_max) / (min(water_density / oil_density, 1.0) * (h * h)))
    cv = c_f + 0.0
    cfl = 0.5 * (cv + math.sqrt((cv * cv + 4.0 * (g_f * g_f)) + 4.0 * (s_f * s_f)))
    return 1.0 / cfl


def pipe_step(phi, u, v, w, grids, C, dt, P):
    """EULERIAN_FLUID_SOLVER_3D::AdvanceOneTimeStepThread of a vertical pipe
    with order_for_time_advancing = 2 and the sourcing step off
    (EULERIAN_FLUID_SOLVER_3D.h:886-979, SolveForRK :1453-1476): the level
    set by Heun over two WENO5 advections (each zeroing u and w outside the
    pipe), the velocity by Heun over two stages of ENO3 advection, body force
    and projection (the pressure of the first stage is the second's initial
    guess), the reinitialisation by Heun over two blocks.  P: tolerance,
    max_iteration, water_density, oil_density, gravity_y, epsilon,
    reinit_iterations, reinit_scaling, p0 (optional), sourcing (optional:
    True runs the reference's Sourcing step, the pipe's semi-implicit
    viscosity, between the body force and the projection, :1466-1469, 2076-
    2100; the object list's sourcing leaves the fields alone for a pipe
    whose only object is the water).  Returns (phi, u, v, w, p)."""
    a = C["a"]
    fixed = pipe_fixed_faces((phi.shape[2], phi.shape[1], phi.shape[0]))
    ph1, u, v, w = pipe_weno5_levelset(phi, u, v, w, grids, a, dt, P["epsilon"])
    ph2, u, v, w = pipe_weno5_levelset(ph1, u, v, w, grids, a, dt, P["epsilon"])
    phi = 0.5 * (phi + ph2)
    rk = (u, v, w)
    p = P.get("p0")
    for _ in range(2):
        u, v, w = pipe_eno3_velocity(u, v, w, grids, a, dt)
        v = pipe_forcing(phi, v, grids, C, P["gravity_y"], P["oil_density"], dt, fixed_v=fixed[1])
        if P.get("sourcing"):
            u, v, w, _vinfo = pipe_viscosity(phi, u, v, w, grids, C, dt, P["tolerance"], P["max_iteration"], fixed)
        u, v, w, p, _info = pipe_projection(phi, u, v, w, grids, C, dt, P["tolerance"], P["max_iteration"],
                                            P["water_density"], P["oil_density"], fixed=fixed, p0=p)
    u, v, w = (0.5 * rk[0] + 0.5 * u, 0.5 * rk[1] + 0.5 * v, 0.5 * rk[2] + 0.5 * w)
    r1 = pipe_reinitialization(phi, grids, P["reinit_iterations"], P["reinit_scaling"], P["epsilon"])
    r2 = pipe_reinitialization(r1, grids, P["reinit_iterations"], P["reinit_scaling"], P["epsilon"])
    phi = 0.5 * (phi + r2)
    return phi, u, v, w, p


# ----------------------------------------------------------------------------
# Oil/water pipe mode, vertical pipe: the semi-implicit viscosity
# (VISCOSITY_3D.h:565-990, 1234-1547, 2048-2300; POISSON_SOLVER_3D.h:342-378,
# 3641-3828)
# ----------------------------------------------------------------------------

def _pipe_visc_copies(comp, b, axis):
    """The velocity copies SetupBoundaryConditionsForVelocity makes for the
    pipe's viscosity (VISCOSITY_3D.h:2048-2300), one component: the masked
    periodic copy `gen` and the copies guarded along x (`cx`) and z (`cz`).
    On faces outside the pipe the guarded copies follow one if/else chain:
    all four transverse neighbours outside -> both 0; else an inside x-1
    (x+1) neighbour gives cx the extrapolation (theta-1)/theta of that
    neighbour; else an inside z-1 (z+1) neighbour gives cz the same; else
    both 0.  The neighbour's value is the masked copy's (the y component
    reads its raw velocity instead, :2166-2200).  Ghosted arrays (G)."""
    g = G
    gen = _pipe_periodic_copy(comp, b, axis == 1)
    src = np.pad(comp, g) if axis == 1 else gen
    cx, cz = gen.copy(), gen.copy()
    nz, ny, nx = b.shape
    bp = np.pad(b, 1)
    c = (slice(1, -1),) * 3

    def bn(ax, s):
        sl = list(c)
        sl[ax] = slice(1 + s, bp.shape[ax] - 1 + s)
        return bp[tuple(sl)]

    def vn(ax, s):
        sl = [slice(g, g + nz), slice(g, g + ny), slice(g, g + nx)]
        sl[ax] = slice(g + s, g + s + b.shape[ax])
        return src[tuple(sl)]

    def ext(bnb, val):
        with np.errstate(divide="ignore", invalid="ignore"):
            theta = np.abs(bnb) / (np.abs(bnb) + np.abs(b))
            return (theta - 1.0) / theta * val

    out = b > 0
    all4 = (bn(2, -1) > 0) & (bn(2, 1) > 0) & (bn(0, -1) > 0) & (bn(0, 1) > 0)
    xm, xp, zm, zp = bn(2, -1) < 0, bn(2, 1) < 0, bn(0, -1) < 0, bn(0, 1) < 0
    ix = (slice(g, g + nz), slice(g, g + ny), slice(g, g + nx))
    cxi, czi = cx[ix], cz[ix]
    new_x = np.where(out & all4, 0.0, cxi)
    new_z = np.where(out & all4, 0.0, czi)
    r1 = out & ~all4 & xm
    r2 = out & ~all4 & ~xm & xp
    r3 = out & ~all4 & ~xm & ~xp & zm
    r4 = out & ~all4 & ~xm & ~xp & ~zm & zp
    r5 = out & ~all4 & ~xm & ~xp & ~zm & ~zp
    new_x = np.where(r1, ext(bn(2, -1), vn(2, -1)), new_x)
    new_x = np.where(r2, ext(bn(2, 1), vn(2, 1)), new_x)
    new_z = np.where(r3, ext(bn(0, -1), vn(0, -1)), new_z)
    new_z = np.where(r4, ext(bn(0, 1), vn(0, 1)), new_z)
    new_x = np.where(r5, 0.0, new_x)
    new_z = np.where(r5, 0.0, new_z)
    cx[ix] = new_x
    cz[ix] = new_z
    return gen, cx, cz


def _shifted(a, ax, s, fill=0.0):
    """a shifted so that out[idx] = a[idx + s e_ax], `fill` beyond the array."""
    out = np.full_like(a, fill)
    src = [slice(None)] * 3
    dst = [slice(None)] * 3
    if s > 0:
        src[ax], dst[ax] = slice(s, None), slice(0, -s)
    else:
        src[ax], dst[ax] = slice(0, s), slice(-s, None)
    out[tuple(dst)] = a[tuple(src)]
    return out


def pipe_viscosity_system(comp, b, axis, coefs, explicit, gen, dx_copy, dz_copy, dx, tol, max_iter, fixed=None):
    """One component of the pipe's semi-implicit solve (SolveForViscosity,
    POISSON_SOLVER_3D.h:342-378, with BuildLinearSystemNodeForSemiImplicit-
    Viscosity :3641-3828 and the boundary tags of SetupBoundaryConditions-
    ForVelocity, VISCOSITY_3D.h:1350-1547).  Unknowns: faces inside the pipe
    (wall distance <= 0) with 0 <= j < ny; faces outside are Dirichlet, the
    rows beyond the ends periodic (row -1 is row ny-2, row ny is row 1, for
    every component).  Row: (1 + sum(coef)/dx^2) x_c - sum coef_n/dx^2 x_n,
    the sum in the reference's order (unknown neighbours l, r, b, t, d, u,
    then periodic b, t, then Dirichlet l, r, d, u; a zero sum becomes 1);
    right-hand side the explicit term plus the Dirichlet neighbours'
    coef/dx^2 times their guarded copies (dx_copy along x, dz_copy along z);
    initial guess the masked copy; the reference's PCG (asymmetric matrix,
    absolute r.z < tol^2).  The solution is written back to every unknown
    but the fixed faces (VectorToGrid, POISSON_SOLVER_3D.h:4060-4077, skips
    faces Solve_Velocity marked fixed).  Returns (new component,
    iterations)."""
    g = G
    c1, c2, c3, c4, c5, c6 = coefs
    nz, ny, nx = b.shape
    jrows = np.arange(ny)[None, :, None]
    rows = (b <= 0) & (jrows < (ny - 1 if axis == 1 else ny))
    inv2 = 1.0 / (dx * dx)
    zero = np.zeros_like(b)
    l_full, r_full = _shifted(rows, 2, -1, False) & rows, _shifted(rows, 2, 1, False) & rows
    d_full, u_full = _shifted(rows, 0, -1, False) & rows, _shifted(rows, 0, 1, False) & rows
    b_full = rows & (jrows > 0)
    t_full = rows & (jrows < ny - (2 if axis == 1 else 1))
    b_per = rows & (jrows == 0)
    t_per = rows & (jrows == ny - (2 if axis == 1 else 1))
    l_dir, r_dir = rows & (_shifted(b, 2, -1) > 0), rows & (_shifted(b, 2, 1) > 0)
    d_dir, u_dir = rows & (_shifted(b, 0, -1) > 0), rows & (_shifted(b, 0, 1) > 0)
    coef = zero
    for m, cv in ((l_full, c2), (r_full, c1), (b_full, c4), (t_full, c3), (d_full, c6), (u_full, c5),
                  (b_per, c4), (t_per, c3), (l_dir, c2), (r_dir, c1), (d_dir, c6), (u_dir, c5)):
        coef = coef + np.where(m, cv, 0.0)
    coef = np.where(rows & (coef == 0), 1.0, coef)
    diag = np.where(rows, 1.0 + inv2 * coef, 1.0)
    ix = (slice(g, g + nz), slice(g, g + ny), slice(g, g + nx))
    vx, vz = dx_copy, dz_copy

    def nbv(a, ax, s):
        sl = list(ix)
        sl[ax] = slice(ix[ax].start + s, ix[ax].stop + s)
        return a[tuple(sl)]

    rhs = np.where(rows, explicit, 0.0)
    for m, cv, val in ((l_dir, c2, nbv(vx, 2, -1)), (r_dir, c1, nbv(vx, 2, 1)), (d_dir, c6, nbv(vz, 0, -1)),
                       (u_dir, c5, nbv(vz, 0, 1))):
        rhs = np.where(m, rhs + cv * inv2 * val, rhs)
    x0 = np.where(rows, gen[ix], 0.0)
    off = [(l_full, -c2 * inv2, (2, -1)), (r_full, -c1 * inv2, (2, 1)), (b_full, -c4 * inv2, (1, -1)),
           (t_full, -c3 * inv2, (1, 1)), (d_full, -c6 * inv2, (0, -1)), (u_full, -c5 * inv2, (0, 1))]
    jb = ny - 2 if axis != 1 else ny - 3  # the periodic images of rows -1 and ny-1+1

    def apply(x):
        q = np.zeros_like(x)
        for m, val, (ax, s) in off:
            q = q + np.where(m, val * _shifted(x, ax, s), 0.0)
        q = q + np.where(b_per, (-c4 * inv2) * np.broadcast_to(x[:, jb:jb + 1, :], x.shape), 0.0)
        q = q + np.where(t_per, (-c3 * inv2) * np.broadcast_to(x[:, 1:2, :], x.shape), 0.0)
        return q + diag * x

    x, it, _rz, _rel = pcg(apply, diag, rhs, x0, tol, max_iter, "abs")
    keep = ~rows if fixed is None else (~rows | fixed)
    out = np.where(keep, comp, x)
    if axis == 1:
        out[:, ny - 1, :] = out[:, 1, :]
    return out, it


def pipe_viscosity(phi, u, v, w, grids, C, dt, tol, max_iter, fixed=None):
    """VISCOSITY_3D::ApplyViscosity of a vertical pipe, the oil/water
    semi-implicit branch in the dimensionless form (VISCOSITY_3D.h:565-990),
    epsilon 1.5 dx (EULERIAN_FLUID_SOLVER_3D.h:394).  Per component, from
    the velocity copies made before any component is solved: smeared
    density rho = 1 + (eta - 1) H and viscosity mu = 1 + (m - 1) H (H the
    viscosity's Heaviside, :1234-1350) of face and edge averages of the
    periodic level set; coef_q = dt/(Re rho) mu (2 dt/(Re rho) mu along the
    component's own axis); the explicit cross terms; then the implicit solve
    (pipe_viscosity_system); `fixed` (per component, optional) are the
    faces Solve_Velocity marked fixed, which keep their value.  Returns
    (u, v, w, info)."""
    g = G
    dx = grids[0][3]
    idx = idy = idz = 1.0 / dx
    eps = 1.5 * dx
    Re, m, eta = C["Re"], C["m"], C["eta"]
    comps = (u, v, w)
    bs = [pipe_boundary(grids[1 + a], comps[a].shape, C["a"]) for a in range(3)]
    cp = [_pipe_visc_copies(comps[a], bs[a], a) for a in range(3)]  # (gen, cx, cz)
    wa = periodic_ghosts_y(phi)
    H = lambda x: heaviside_viscosity(x, eps)
    rho_of = lambda x: 1.0 + (eta - 1.0) * H(x)
    mu_of = lambda x: 1.0 + (m - 1.0) * H(x)
    nzc, nyc, nxc = phi.shape
    out, info = [], {}
    for a in range(3):
        sh = comps[a].shape

        def W(di, dj, dk):
            return wa[g + dk:g + dk + sh[0], g + dj:g + dj + sh[1], g + di:g + di + sh[2]]

        def F(arr, di, dj, dk, shape):  # a ghosted face copy at the offset, on this component's face grid
            return arr[g + dk:g + dk + sh[0], g + dj:g + dj + sh[1], g + di:g + di + sh[2]]

        if a == 0:
            lo, hi = W(-1, 0, 0), W(0, 0, 0)
            half = 0.5 * (lo + hi)
            e1 = 0.25 * (((lo + hi) + W(-1, 1, 0)) + W(0, 1, 0))   # cu
            e2 = 0.25 * (((lo + hi) + W(-1, -1, 0)) + W(0, -1, 0))  # cd
            e3 = 0.25 * (((lo + hi) + W(-1, 0, 1)) + W(0, 0, 1))   # ct
            e4 = 0.25 * (((lo + hi) + W(-1, 0, -1)) + W(0, 0, -1))  # cb
            rho = rho_of(half)
            mu_r, mu_c, mu_cu, mu_cd, mu_ct, mu_cb = (mu_of(x) for x in (hi, lo, e1, e2, e3, e4))
            A, A2 = dt / (Re * rho), (2.0 * dt) / (Re * rho)
            coefs = (A2 * mu_r, A2 * mu_c, A * mu_cu, A * mu_cd, A * mu_ct, A * mu_cb)
            yx, zx = cp[1][1], cp[2][1]
            ex = F(cp[0][0], 0, 0, 0, sh) + A * (idy * (mu_cu * idx * (F(yx, 0, 1, 0, sh) - F(yx, -1, 1, 0, sh))
                                                      - mu_cd * idx * (F(yx, 0, 0, 0, sh) - F(yx, -1, 0, 0, sh))))
            ex = ex + A * (idz * (mu_ct * idx * (F(zx, 0, 0, 1, sh) - F(zx, -1, 0, 1, sh))
                                  - mu_cb * idx * (F(zx, 0, 0, 0, sh) - F(zx, -1, 0, 0, sh))))
        elif a == 1:
            lo, hi = W(0, -1, 0), W(0, 0, 0)
            half = 0.5 * (lo + hi)
            e1 = 0.25 * (((lo + W(1, -1, 0)) + hi) + W(1, 0, 0))             # cu
            e2 = 0.25 * (((W(-1, -1, 0) + lo) + W(-1, 0, 0)) + hi)           # cl
            e3 = 0.25 * (((W(0, -1, 1) + lo) + W(0, 0, 1)) + hi)             # ct
            e4 = 0.25 * (((W(0, -1, -1) + lo) + W(0, 0, -1)) + hi)           # cb
            rho = rho_of(half)
            mu_cu, mu_cl, mu_u, mu_c, mu_ct, mu_cb = (mu_of(x) for x in (e1, e2, hi, lo, e3, e4))
            A, A2 = dt / (Re * rho), (2.0 * dt) / (Re * rho)
            coefs = (A * mu_cu, A * mu_cl, A2 * mu_u, A2 * mu_c, A * mu_ct, A * mu_cb)
            xx, zz = cp[0][1], cp[2][2]
            ex = F(cp[1][0], 0, 0, 0, sh) + A * (idx * (mu_cu * idy * (F(xx, 1, 0, 0, sh) - F(xx, 1, -1, 0, sh))
                                                      - mu_cl * idy * (F(xx, 0, 0, 0, sh) - F(xx, 0, -1, 0, sh))))
            ex = ex + A * (idz * (mu_ct * idy * (F(zz, 0, 0, 1, sh) - F(zz, 0, -1, 1, sh))
                                  - mu_cb * idx * (F(zz, 0, 0, 0, sh) - F(zz, 0, -1, 0, sh))))
        else:
            lo, hi = W(0, 0, -1), W(0, 0, 0)
            half = 0.5 * (lo + hi)
            e1 = 0.25 * (((lo + W(1, 0, -1)) + hi) + W(1, 0, 0))    # ct
            e2 = 0.25 * (((lo + W(-1, 0, -1)) + hi) + W(-1, 0, 0))  # cb
            e3 = 0.25 * (((lo + W(0, 1, -1)) + hi) + W(0, 1, 0))    # cu
            e4 = 0.25 * (((lo + W(0, -1, -1)) + hi) + W(0, -1, 0))  # cd
            rho = rho_of(half)
            mu_ct, mu_cb, mu_cu, mu_cd, mu_t, mu_c = (mu_of(x) for x in (e1, e2, e3, e4, hi, lo))
            A, A2 = dt / (Re * rho), (2.0 * dt) / (Re * rho)
            coefs = (A * mu_ct, A * mu_cb, A * mu_cu, A * mu_cd, A2 * mu_t, A2 * mu_c)
            xz, yz = cp[0][2], cp[1][2]
            ex = F(cp[2][0], 0, 0, 0, sh) + A * (idx * (idz * (mu_ct * (F(xz, 1, 0, 0, sh) - F(xz, 1, 0, -1, sh)))
                                                      - idz * (mu_cb * (F(xz, 0, 0, 0, sh) - F(xz, 0, 0, -1, sh)))))
            ex = ex + A * (idy * (idz * (mu_cu * (F(yz, 0, 1, 0, sh) - F(yz, 0, 1, -1, sh)))
                                  - idz * (mu_cd * (F(yz, 0, 0, 0, sh) - F(yz, 0, 0, -1, sh)))))
        gen, cx, cz = cp[a]
        new, it = pipe_viscosity_system(comps[a], bs[a], a, coefs, ex, gen, cx, cz, dx, tol, max_iter,
                                        None if fixed is None else fixed[a])
        out.append(new)
        info[f"coef_{'uvw'[a]}"] = coefs
        info[f"explicit_{'uvw'[a]}"] = ex
        info[f"iterations_{'uvw'[a]}"] = it
    return out[0], out[1], out[2], info
