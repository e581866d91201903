"""b2s_spmv_noalloc: the SpMV entry point for callers that cannot allocate.

Some callers cannot call cudaMalloc (they run inside a host callback or an
allocator hook, or live in a process whose device memory belongs to another
framework's caching allocator). They own the matrix and vectors; the entry
point allocates nothing and keeps its small scratch in a fixed device array.
This file is named so that pytest collects it last. It checks two calls in a
row against the existing b2s_spmv (same tolerance as the SpMV parity test:
1e-13 relative in y, 1e-12 in the dot), and the size limit.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import to_dev

pytestmark = pytest.mark.gpu

MAX_BLOCKS = 8_388_608


def _noalloc(lib, nb, rows, cols, vals, x, y, dot, stream=None):
    return lib.b2s_spmv_noalloc(nb, int(rows.numel()), C.c_void_p(rows.data_ptr()), C.c_void_p(cols.data_ptr()),
                                C.c_void_p(vals.data_ptr()), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                C.c_void_p(dot.data_ptr()) if dot is not None else None, stream)


def test_noalloc_spmv_matches_b2s_spmv_twice(solver, cuda, stack_small):
    import torch

    s = stack_small
    solver.assemble(s.n_verts, to_dev(s.rows, cuda), to_dev(s.cols, cuda), to_dev(s.vals, cuda))
    rowptr, col, val = solver.upper_bsr()
    rows = np.repeat(np.arange(s.n_verts, dtype=np.int32), np.diff(rowptr))
    d_rows, d_cols = to_dev(rows, cuda), to_dev(col, cuda)
    d_vals = to_dev(val, cuda)  # [nnz, 9] column-major blocks
    lib = solver.lib
    rng = np.random.default_rng(21)
    for call in range(2):
        x = to_dev(rng.standard_normal(3 * s.n_verts), cuda)
        y_ref = torch.empty_like(x)
        dot_ref = solver.spmv(x, y_ref, with_dot=True)
        y = torch.full_like(x, float("nan"))  # every entry must be overwritten
        dot = torch.zeros(1, dtype=torch.float64, device=cuda)
        rc = _noalloc(lib, s.n_verts, d_rows, d_cols, d_vals, x, y, dot)
        assert rc == 0, lib.b2s_last_error(None).decode()
        torch.cuda.synchronize()
        yr = y_ref.cpu().numpy()
        assert np.abs(y.cpu().numpy() - yr).max() <= 1e-13 * np.abs(yr).max(), f"call {call}"
        assert abs(float(dot.item()) - dot_ref) <= 1e-12 * abs(dot_ref), f"call {call}"


def test_noalloc_spmv_rejects_oversized_input(cuda):
    from libuipc_b200._native import load_solve_lib

    lib = load_solve_lib()
    one = C.c_void_p(1)  # never dereferenced: the size check comes first
    rc = lib.b2s_spmv_noalloc(1, MAX_BLOCKS + 1, one, one, one, one, one, None, None)
    assert rc == -1
    assert b"limit" in lib.b2s_last_error(None)
