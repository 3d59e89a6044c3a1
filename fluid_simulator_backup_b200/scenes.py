"""The synthetic scenes of the benchmark configurations, as FP64 arrays in
the library's layout ([z, y, x], x fastest; faces [n, n, n+1], [n, n+1, n],
[n+1, n, n]), and the smeared-Heaviside volume the reference uses for its
phase volumes (EULERIAN_FLUID_SOLVER_3D.h:2459-2479, eps = 1.5 dx)."""
import numpy as np


def axes(n):
    x = (np.arange(n) + 0.5) / n
    return x[None, None, :], x[None, :, None], x[:, None, None]


def zero_faces(n):
    return np.zeros((n, n, n + 1)), np.zeros((n, n + 1, n)), np.zeros((n + 1, n, n))


def dam_break(n):
    """Signed distance to the water box [0,0.4] x [0,0.6] x [0,1] on the unit
    cube, negative inside."""
    x, y, z = axes(n)
    lo, hi = np.array([0.0, 0.0, 0.0]), np.array([0.4, 0.6, 1.0])
    d = np.broadcast_arrays(*[np.maximum(lo[a] - c, c - hi[a]) for a, c in enumerate((x, y, z))])
    outside = np.sqrt(sum(np.maximum(q, 0.0) ** 2 for q in d))
    inside = np.minimum(np.maximum(np.maximum(d[0], d[1]), d[2]), 0.0)
    return outside + inside


def rising_bubble(n, radius=0.15, centre=(0.5, 0.25, 0.5)):
    """Signed distance to an air sphere (negative inside) in water."""
    x, y, z = axes(n)
    return np.sqrt((x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2) - radius


def rayleigh_taylor(n, seed=0):
    """y - 0.5 minus a perturbation of amplitude 0.01 made of the modes
    kx, kz in 1..8 with amplitudes N(0, 1) and phases U(0, 1) drawn from
    default_rng(seed); negative below the interface (the light phase)."""
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


def heaviside_volume(phi, dx):
    """Volume of the phase phi < 0: sum of H(-phi) dx^3 with the smeared
    Heaviside H(x) = 0 (x < -eps), 1 (x > eps), 1/2 + x/(2 eps) +
    sin(pi x / eps)/(2 pi) between, eps = 1.5 dx."""
    eps = 1.5 * dx
    x = -phi
    h = np.where(x < -eps, 0.0, np.where(x > eps, 1.0, 0.5 + x / (2 * eps) + np.sin(np.pi * x / eps) / (2 * np.pi)))
    return float(h.sum()) * dx ** 3
