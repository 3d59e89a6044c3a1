"""fs_pcg_csr_noalloc: the allocation-free CSR Jacobi-PCG entry point.

Collected last (file name) so that it also runs after every other test has
used the library on the same device.  Each call goes through the C ABI with
device pointers the test owns and is compared with fs_pcg_csr, the
allocating entry point, on the same system.
"""
import ctypes
import os

import numpy as np
import pytest

import fluid_simulator_backup_b200 as fs

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
MAX_ROWS = 1 << 18


def variable_poisson_csr(n, seed):
    """7-point SPD system on an n^3 grid: random positive face couplings,
    diagonal = sum of couplings + a small shift; rows in (k, j, i) order."""
    rng = np.random.default_rng(seed)
    N = n ** 3
    idx = np.arange(N).reshape(n, n, n)
    rows, cols, vals = [], [], []
    diag = np.full(N, 0.05)
    for axis in range(3):
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[axis] = slice(0, n - 1)
        hi[axis] = slice(1, n)
        a = idx[tuple(lo)].ravel()
        c = idx[tuple(hi)].ravel()
        coef = rng.uniform(0.5, 2.0, a.size) * (10.0 if axis == 2 else 1.0)
        rows += [a, c]
        cols += [c, a]
        vals += [-coef, -coef]
        np.add.at(diag, a, coef)
        np.add.at(diag, c, coef)
    rows.append(np.arange(N))
    cols.append(np.arange(N))
    vals.append(diag)
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    vals = np.concatenate(vals)
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    rowptr = np.zeros(N + 1, dtype=np.int32)
    np.add.at(rowptr, rows + 1, 1)
    rowptr = np.cumsum(rowptr).astype(np.int32)
    b = rng.standard_normal(N)
    return vals, cols.astype(np.int32), rowptr, b


def noalloc_solve(torch, vals, cols, rowptr, b, tol, max_iter, stop, stream=None):
    dev = torch.device("cuda:0")
    dv = torch.from_numpy(np.ascontiguousarray(vals, np.float64)).to(dev)
    dc = torch.from_numpy(np.ascontiguousarray(cols, np.int32)).to(dev)
    dr = torch.from_numpy(np.ascontiguousarray(rowptr, np.int32)).to(dev)
    db = torch.from_numpy(np.ascontiguousarray(b, np.float64)).to(dev)
    dx = torch.zeros_like(db)
    torch.cuda.synchronize()
    it = ctypes.c_int()
    res = ctypes.c_double()
    handle = stream.cuda_stream if stream is not None else None
    status = fs.lib().fs_pcg_csr_noalloc(len(b), len(vals), dv.data_ptr(), dc.data_ptr(), dr.data_ptr(),
                                         db.data_ptr(), dx.data_ptr(), float(tol), int(max_iter), int(stop),
                                         handle, ctypes.byref(it), ctypes.byref(res))
    torch.cuda.synchronize()
    return dx.cpu().numpy(), it.value, res.value, status


def csr_residual(vals, cols, rowptr, b, x):
    rows = np.repeat(np.arange(len(b)), np.diff(rowptr))
    ax = np.bincount(rows, weights=vals * x[cols], minlength=len(b))
    return float(np.linalg.norm(b - ax) / np.linalg.norm(b))


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.gpu
def test_noalloc_matches_allocating_solver_two_calls_in_a_row():
    import torch

    g = np.load(os.path.join(GOLDEN, "projection_bubble.npz"))
    first = (g["csr_vals"], g["csr_cols"], g["csr_rowptr"], g["b"], float(g["tol"]), fs.FS_STOP_ABSOLUTE)
    second = variable_poisson_csr(48, 3) + (1e-12, fs.FS_STOP_RELATIVE)
    side = torch.cuda.Stream()
    for case, stream in ((first, None), (second, side), (first, side)):
        vals, cols, rowptr, b, tol, stop = case
        x_ref, it_ref, res_ref, st_ref = fs.pcg_csr(vals, cols, rowptr, b, np.zeros_like(b), tol, 100000, stop)
        x, it, res, st = noalloc_solve(torch, vals, cols, rowptr, b, tol, 100000, stop, stream)
        assert st == fs.FS_OK == st_ref
        # the two run the same kernels; only the order of the atomic partial
        # sums differs, which may move the stopping iteration by a little
        assert abs(it - it_ref) <= 2 + it_ref // 100
        assert rel(x, x_ref) < 1e-7
        if stop == fs.FS_STOP_RELATIVE:
            assert res <= tol
            assert csr_residual(vals, cols, rowptr, b, x) < 10 * tol
    # the reference's own PCG solution of the first system
    x, it, _, st = noalloc_solve(torch, *first[:4], first[4], 100000, first[5])
    assert st == fs.FS_OK
    assert abs(it - int(g["iterations"])) <= 2
    assert rel(x, g["x"]) < 1e-7


@pytest.mark.gpu
def test_noalloc_reports_iteration_limit_and_rejects_oversize():
    import torch

    vals, cols, rowptr, b = variable_poisson_csr(16, 4)
    x, it, res, st = noalloc_solve(torch, vals, cols, rowptr, b, 1e-14, 5, fs.FS_STOP_RELATIVE)
    assert st == fs.FS_NOT_CONVERGED and it == 5 and np.isfinite(res)
    # more rows than the fixed scratch holds: rejected before any device work
    d = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    st = fs.lib().fs_pcg_csr_noalloc(MAX_ROWS + 1, 7 * (MAX_ROWS + 1), d.data_ptr(), d.data_ptr(), d.data_ptr(),
                                     d.data_ptr(), d.data_ptr(), 1e-6, 10, fs.FS_STOP_RELATIVE, None, None, None)
    assert st == fs.FS_INVALID_ARG


@pytest.mark.gpu
def test_noalloc_rejects_out_of_range_indices_on_the_device():
    """A column index outside [0, n) or a row_ptr entry beyond nnz is found by
    the device-side check before the matrix is used: FS_INVALID_ARG, x left
    as it came, and the next call on a valid system is unaffected."""
    import torch

    vals, cols, rowptr, b = variable_poisson_csr(8, 5)
    bad_col = cols.copy()
    bad_col[17] = len(b)  # one past the last row
    bad_ptr = rowptr.copy()
    bad_ptr[5] = len(vals) + 3  # beyond nnz (and decreasing after it)
    for c, r in ((bad_col, rowptr), (cols, bad_ptr)):
        x, it, res, st = noalloc_solve(torch, vals, c, r, b, 1e-10, 100, fs.FS_STOP_RELATIVE)
        assert st == fs.FS_INVALID_ARG
        assert not np.any(x)  # the zero initial guess is untouched
    x, it, res, st = noalloc_solve(torch, vals, cols, rowptr, b, 1e-10, 1000, fs.FS_STOP_RELATIVE)
    assert st == fs.FS_OK and res <= 1e-10


@pytest.mark.gpu
def test_zero_iteration_cap_runs_no_iteration():
    """max_iteration = 0 runs no iteration, as PCG_METHOD::PCGMethod's
    `while (num_iteration < max_iteration)` loop (PCG_METHOD.cpp:4-126): x is
    unchanged and the solve reports 0 iterations, in both CSR entry points."""
    import torch

    vals, cols, rowptr, b = variable_poisson_csr(8, 6)
    x0 = np.full_like(b, 0.25)
    x, it, res, st = fs.pcg_csr(vals, cols, rowptr, b, x0, 1e-10, 0, fs.FS_STOP_RELATIVE)
    assert st == fs.FS_NOT_CONVERGED and it == 0
    np.testing.assert_array_equal(x, x0)
    x, it, res, st = noalloc_solve(torch, vals, cols, rowptr, b, 1e-10, 0, fs.FS_STOP_RELATIVE)
    assert st == fs.FS_NOT_CONVERGED and it == 0 and not np.any(x)
