"""The zero level set as a triangle mesh (WRITE_LEVELSET::WriteOBJ,
WRITE_LEVELSET.h:22-84; MARCHING_CUBES_ALGORITHM.h) through the C ABI on the
GPU: FP64 vertices and triangles bit for bit equal to the oracle's marching
cubes (normals to 1e-10: they are summed in 2^-40 fixed point), FP32 storage to its
rounding, the reference's own surfaces (golden) by the same properties the
oracle meets, and the OBJ file."""
import os

import numpy as np
import pytest

import fluid_simulator_backup_b200 as fs
from oracle import fs_oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
pytestmark = pytest.mark.gpu


def noisy_sphere(n, seed, c=(0.5, 0.45, 0.4), r=0.3, scale=1.3, noise=0.002):
    nx, ny, nz = n
    dx = 1.0 / nx
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dx
    z = (np.arange(nz) + 0.5) * dx
    sd = np.sqrt((x[None, None, :] - c[0]) ** 2 + (y[None, :, None] - c[1]) ** 2 + (z[:, None, None] - c[2]) ** 2) - r
    return sd * scale + np.random.default_rng(seed).normal(size=sd.shape) * noise


def gpu_surface(phi, dx, precision=fs.FS_PRECISION_FP64):
    nz, ny, nx = phi.shape
    with fs.Solver((nx, ny, nz), dx, precision=precision) as s:
        s.upload("phi", phi)
        return s.surface()


@pytest.mark.parametrize("n", [(20, 24, 18), (32, 32, 32)])
def test_surface_matches_the_oracle_bit_for_bit(n):
    phi = noisy_sphere(n, 3)
    dx = 1.0 / n[0]
    xyz, nrm, tri = gpu_surface(phi, dx)
    rx, rn, rt = O.marching_cubes(phi, dx)
    np.testing.assert_array_equal(xyz, rx)
    np.testing.assert_array_equal(tri, rt)
    assert np.abs(nrm - rn).max() < 1e-10


def test_two_bodies_touching_the_walls():
    """Two blobs, one cut by the box walls: the walls close nothing (the
    mesh stays open there, as the reference's does), the rest matches."""
    n = (24, 20, 22)
    a = noisy_sphere(n, 5, c=(0.3, 0.4, 0.45), r=0.2, scale=1.0, noise=0.0)
    b = noisy_sphere(n, 6, c=(0.95, 0.1, 0.5), r=0.25, scale=1.0, noise=0.0)
    phi = np.minimum(a, b)
    dx = 1.0 / n[0]
    xyz, nrm, tri = gpu_surface(phi, dx)
    rx, rn, rt = O.marching_cubes(phi, dx)
    np.testing.assert_array_equal(xyz, rx)
    np.testing.assert_array_equal(tri, rt)


def test_fp32_surface_is_close():
    n = (24, 24, 24)
    phi = noisy_sphere(n, 7, noise=0.0)
    dx = 1.0 / 24
    xyz, _, tri = gpu_surface(phi, dx, fs.FS_PRECISION_FP32_REFINE)
    rx, _, rt = O.marching_cubes(phi, dx)
    assert xyz.shape == rx.shape and tri.shape == rt.shape
    assert np.abs(xyz - rx).max() < 1e-6


@pytest.mark.parametrize("name", ["surface_sphere", "surface_noisy"])
def test_golden_surface_through_cuda(name):
    from scipy.spatial import cKDTree
    from test_oracle_golden import closed_and_oriented, mesh_area, mesh_volume
    g = dict(np.load(os.path.join(GOLD, name + ".npz")))
    xyz, nrm, tri = gpu_surface(g["phi"], float(g["dx"]))
    assert xyz.shape == g["xyz"].shape and tri.shape == g["tri"].shape
    dist, idx = cKDTree(g["xyz"]).query(xyz)
    assert dist.max() <= 2e-15 and len(set(idx.tolist())) == len(idx)
    assert abs(mesh_area(xyz, tri) / mesh_area(g["xyz"], g["tri"]) - 1) < 1e-5
    assert abs(mesh_volume(xyz, tri) / mesh_volume(g["xyz"], g["tri"]) - 1) < 5e-4
    assert closed_and_oriented(tri)
    assert np.all(np.einsum("ij,ij->i", nrm, g["normals"][idx]) > 0.5)


def test_write_obj(tmp_path):
    n = (16, 16, 16)
    phi = noisy_sphere(n, 9, noise=0.0)
    path = str(tmp_path / "surface.obj")
    with fs.Solver(n, 1.0 / 16) as s:
        s.upload("phi", phi)
        s.write_obj(path)
        xyz, nrm, tri = s.surface()
    v, vn, f = [], [], []
    for line in open(path):
        head, *rest = line.split()
        if head == "v":
            v.append([float(t) for t in rest])
        elif head == "vn":
            vn.append([float(t) for t in rest])
        elif head == "f":
            f.append([int(t.split("//")[0]) for t in rest])
            assert all(t.split("//")[0] == t.split("//")[1] for t in rest)
    np.testing.assert_allclose(np.array(v), xyz, rtol=1e-8, atol=1e-9)
    np.testing.assert_allclose(np.array(vn), nrm, rtol=1e-8, atol=1e-9)
    np.testing.assert_array_equal(np.array(f), tri)


def test_surface_is_deterministic():
    """Two extractions of the same level set give the same bits, normals
    included (order-independent integer sums)."""
    n = (24, 24, 24)
    phi = noisy_sphere(n, 12)
    a = gpu_surface(phi, 1.0 / 24)
    b = gpu_surface(phi, 1.0 / 24)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_empty_surface():
    with fs.Solver((12, 12, 12), 1.0 / 12) as s:
        s.upload("phi", np.ones((12, 12, 12)))
        xyz, nrm, tri = s.surface()
    assert xyz.shape == (0, 3) and tri.shape == (0, 3)
