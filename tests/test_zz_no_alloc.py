"""prism_jacobi_step_noalloc: the Jacobi sweep for callers that cannot allocate
device memory when they need a solver step (host applications with a fixed
device-memory budget, time loops that must not synchronize on cudaMalloc/cudaFree).
It must give the same result as the allocating entry point, prism_solve_csr with
the Jacobi method, call after call, and as a CPU restatement of the reference's
numerics/jacobi.cpp:5-9 (x + D^-1 (b - A x), D^-1 = 1/diag, inf where a row has
no diagonal entry), up to its largest size.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes when run alone."""
import ctypes

import numpy as np
import pytest

from prism_b200 import PrismError, api
from prism_b200 import _abi as A

pytestmark = pytest.mark.gpu
MAX_ROWS = 1048576  # PRISM_NOALLOC_MAX_ROWS
RTOL = 1e-13


def random_system(n, seed=7):
    """Diagonally dominant sparse matrix with ragged rows (1 to 9 entries), CSR sorted by column."""
    rng = np.random.default_rng(seed)
    k = rng.integers(0, 9, size=n)
    rows = np.repeat(np.arange(n), k)
    cols = rng.integers(0, n, size=rows.size)
    keep = cols != rows
    rows, cols = rows[keep], cols[keep]
    key = np.unique(rows.astype(np.int64) * n + cols)
    rows, cols = key // n, key % n
    off = rng.uniform(-1.0, 1.0, size=rows.size)
    dom = np.bincount(rows, weights=np.abs(off), minlength=n) + rng.uniform(0.5, 2.0, size=n)
    rows = np.concatenate([rows, np.arange(n)])
    cols = np.concatenate([cols, np.arange(n)])
    vals = np.concatenate([off, dom])
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    rowptr = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int64)
    return rowptr, cols.astype(np.int64), vals, rng.normal(size=n), rng.normal(size=n)


def jacobi_cpu(rowptr, col, val, b, x):
    """numerics/jacobi.cpp:5-9 restated with numpy: D_inv = 1 / diag (0 where the row has no
    diagonal entry), r = b - A x, x + D_inv * r."""
    n = len(b)
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    Ax = np.bincount(rows, weights=val * x[col], minlength=n)
    diag = np.bincount(rows[col == rows], weights=val[col == rows], minlength=n)
    with np.errstate(divide="ignore", invalid="ignore"):
        return x + (1.0 / diag) * (b - Ax)


class DeviceCsr:
    """CSR arrays and vectors in device memory owned by the caller (torch), int32 indices."""

    def __init__(self, rowptr, col, val, b, x):
        import torch
        dev = torch.device("cuda")
        self.rowptr = torch.tensor(rowptr.astype(np.int32), device=dev)
        self.col = torch.tensor(col.astype(np.int32), device=dev)
        self.val = torch.tensor(val, device=dev)
        self.b = torch.tensor(b, device=dev)
        self.x = torch.tensor(x, device=dev)
        self.n = len(b)

    def sweep(self, gpu):
        import torch
        stream = torch.cuda.current_stream().cuda_stream
        gpu.check(gpu.jacobi_step_noalloc(self.n, self.rowptr.data_ptr(), self.col.data_ptr(), self.val.data_ptr(),
                                          self.b.data_ptr(), self.x.data_ptr(), ctypes.c_void_p(stream)))
        torch.cuda.synchronize()
        return self.x.cpu().numpy().copy()


def close(a, ref):
    np.testing.assert_allclose(a, ref, rtol=RTOL, atol=RTOL * np.abs(ref[np.isfinite(ref)]).max())


def test_noalloc_matches_allocating_entry_point_and_cpu(gpu):
    n = 5000
    rowptr, col, val, b, x0 = random_system(n)
    d = DeviceCsr(rowptr, col, val, b, x0)
    outs = [d.sweep(gpu), d.sweep(gpu)]  # two calls in a row on the same buffers
    # the allocating entry point, one and two sweeps
    one = api.Jacobi().step(gpu, rowptr, col, val, x0, b)
    two = api.Jacobi().step(gpu, rowptr, col, val, one, b)
    close(outs[0], one)
    close(outs[1], two)
    # the CPU restatement of the reference
    cpu1 = jacobi_cpu(rowptr, col, val, b, x0)
    close(outs[0], cpu1)
    close(outs[1], jacobi_cpu(rowptr, col, val, b, cpu1))


def test_noalloc_row_without_diagonal(gpu):
    # the reference's D^-1 is inf on such a row (x + inf r); the allocating entry point
    # rejects the matrix instead
    n = 64
    rowptr, col, val, b, x0 = random_system(n, seed=3)
    r = 17
    keep = ~((np.repeat(np.arange(n), np.diff(rowptr)) == r) & (col == r))
    lens = np.diff(rowptr).copy()
    lens[r] -= 1
    rowptr2 = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    col2, val2 = col[keep], val[keep]
    out = DeviceCsr(rowptr2, col2, val2, b, x0).sweep(gpu)
    ref = jacobi_cpu(rowptr2, col2, val2, b, x0)
    assert np.isinf(ref[r]) and out[r] == ref[r]
    mask = np.arange(n) != r
    close(out[mask], ref[mask])
    with pytest.raises(PrismError) as e:
        api.Jacobi().step(gpu, rowptr2, col2, val2, x0, b)
    assert e.value.status == A.BAD_ARG


def test_noalloc_largest_size(gpu):
    rowptr, col, val, b, x0 = random_system(MAX_ROWS, seed=11)
    d = DeviceCsr(rowptr, col, val, b, x0)
    out1 = d.sweep(gpu)
    out2 = d.sweep(gpu)
    cpu1 = jacobi_cpu(rowptr, col, val, b, x0)
    close(out1, cpu1)
    close(out2, jacobi_cpu(rowptr, col, val, b, cpu1))


def test_noalloc_rejects_too_many_rows(gpu):
    import torch
    dev = torch.device("cuda")
    dummy = torch.zeros(4, dtype=torch.float64, device=dev)
    idx = torch.zeros(4, dtype=torch.int32, device=dev)
    st = gpu.jacobi_step_noalloc(MAX_ROWS + 1, idx.data_ptr(), idx.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
                                 dummy.data_ptr(), None)
    assert st == A.BAD_ARG
    assert b"exceeds" in gpu.last_error()
