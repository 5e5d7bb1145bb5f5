"""prism_jacobi_step_noalloc: the Jacobi sweep for callers that cannot allocate
device memory (CUDA-graph capture, fixed device-memory budgets, loops that must
not synchronize on cudaMalloc/cudaFree). It must give the same result as the
allocating entry point, prism_solve_csr with the Jacobi method, call after call.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes when run alone."""
import ctypes

import numpy as np
import pytest

from prism_b200 import _abi as A
from prism_b200 import api

pytestmark = pytest.mark.gpu
MAX_ROWS = 1048576  # PRISM_NOALLOC_MAX_ROWS
RTOL = 1e-13


def random_system(n, seed=7):
    # diagonally dominant sparse matrix with ragged rows (1..9 entries)
    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    for i in range(n):
        k = rng.integers(0, 9)
        js = np.unique(rng.integers(0, n, size=k))
        js = js[js != i]
        off = rng.uniform(-1.0, 1.0, size=len(js))
        rows += [i] * (len(js) + 1)
        cols += [i] + list(js)
        vals += [np.abs(off).sum() + rng.uniform(0.5, 2.0)] + list(off)
    order = np.lexsort((np.array(cols), np.array(rows)))
    rows, cols, vals = np.array(rows)[order], np.array(cols)[order], np.array(vals)[order]
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(rowptr, rows + 1, 1)
    rowptr = np.cumsum(rowptr)
    b = rng.normal(size=n)
    x0 = rng.normal(size=n)
    return rowptr, cols.astype(np.int64), vals, b, x0


def test_noalloc_matches_allocating_entry_point(gpu):
    import torch
    n = 5000
    rowptr, col, val, b, x0 = random_system(n)
    # the allocating entry point, two sweeps
    ref = x0.copy()
    for _ in range(2):
        ref = api.Jacobi().step(gpu, rowptr, col, val, ref, b)
    # the allocation-free entry point on device buffers the caller owns, two calls in a row
    dev = torch.device("cuda")
    d_rowptr = torch.tensor(rowptr.astype(np.int32), device=dev)
    d_col = torch.tensor(col.astype(np.int32), device=dev)
    d_val = torch.tensor(val, device=dev)
    d_b = torch.tensor(b, device=dev)
    d_x = torch.tensor(x0, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    outs = []
    for _ in range(2):
        st = gpu.jacobi_step_noalloc(n, d_rowptr.data_ptr(), d_col.data_ptr(), d_val.data_ptr(), d_b.data_ptr(),
                                     d_x.data_ptr(), ctypes.c_void_p(stream))
        gpu.check(st)
        torch.cuda.synchronize()
        outs.append(d_x.cpu().numpy().copy())
    first_ref = api.Jacobi().step(gpu, rowptr, col, val, x0, b)
    np.testing.assert_allclose(outs[0], first_ref, rtol=RTOL, atol=RTOL * np.abs(first_ref).max())
    np.testing.assert_allclose(outs[1], ref, rtol=RTOL, atol=RTOL * np.abs(ref).max())


def test_noalloc_rejects_too_many_rows(gpu):
    import torch
    dev = torch.device("cuda")
    dummy = torch.zeros(4, dtype=torch.float64, device=dev)
    idx = torch.zeros(4, dtype=torch.int32, device=dev)
    st = gpu.jacobi_step_noalloc(MAX_ROWS + 1, idx.data_ptr(), idx.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
                                 dummy.data_ptr(), None)
    assert st == A.BAD_ARG
    assert b"exceeds" in gpu.last_error()
