"""b2s_spmv_noalloc: the SpMV entry point for callers that cannot allocate.

Some callers cannot call cudaMalloc (they run inside a host callback or an
allocator hook, or live in a process whose device memory belongs to another
framework's caching allocator). They own the matrix and vectors; the entry
point allocates nothing and keeps its small scratch in a fixed device array.
This file is named so that pytest collects it last. It checks two calls in a
row against the oracle's symmetric SpMV (Spmv::cpu_sym_spmv restated) and
against the existing b2s_spmv (1e-13 relative in y, 1e-12 in the dot), the
size limit, and that malformed input (a column out of range, rows out of
order) is skipped by the kernel's own checks and reported as a NaN dot.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import to_dev
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MAX_BLOCKS = 8_388_608


def _noalloc(lib, nb, rows, cols, vals, x, y, dot, stream=None):
    return lib.b2s_spmv_noalloc(nb, int(rows.numel()), C.c_void_p(rows.data_ptr()), C.c_void_p(cols.data_ptr()),
                                C.c_void_p(vals.data_ptr()), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                C.c_void_p(dot.data_ptr()) if dot is not None else None, stream)


def _bcoo(solver, s, cuda):
    solver.assemble(s.n_verts, to_dev(s.rows, cuda), to_dev(s.cols, cuda), to_dev(s.vals, cuda))
    rowptr, col, val = solver.upper_bsr()
    rows = np.repeat(np.arange(s.n_verts, dtype=np.int32), np.diff(rowptr))
    return rows, col, val


def test_noalloc_spmv_matches_oracle_and_b2s_spmv_twice(solver, cuda, stack_small):
    import torch

    s = stack_small
    rows, col, val = _bcoo(solver, s, cuda)
    d_rows, d_cols = to_dev(rows, cuda), to_dev(col, cuda)
    d_vals = to_dev(val, cuda)  # [nnz, 9] column-major blocks
    A = O.OracleMatrix(s.n_verts, s.rows, s.cols, s.vals)
    lib = solver.lib
    rng = np.random.default_rng(21)
    for call in range(2):
        xh = rng.standard_normal(3 * s.n_verts)
        x = to_dev(xh, cuda)
        y = torch.full_like(x, float("nan"))  # every entry must be overwritten
        dot = torch.zeros(1, dtype=torch.float64, device=cuda)
        rc = _noalloc(lib, s.n_verts, d_rows, d_cols, d_vals, x, y, dot)
        assert rc == 0, lib.b2s_last_error(None).decode()
        torch.cuda.synchronize()
        yg = y.cpu().numpy()
        yo = A.spmv(xh)
        assert np.abs(yg - yo).max() <= 1e-13 * np.abs(yo).max(), f"call {call}"
        do = float(xh @ yo)
        assert abs(float(dot.item()) - do) <= 1e-12 * abs(do), f"call {call}"
        y_ref = torch.empty_like(x)
        dot_ref = solver.spmv(x, y_ref, with_dot=True)
        assert np.abs(yg - y_ref.cpu().numpy()).max() <= 1e-13 * np.abs(yo).max(), f"call {call}"
        assert abs(float(dot.item()) - dot_ref) <= 1e-12 * abs(dot_ref), f"call {call}"


def test_noalloc_spmv_flags_malformed_input(solver, cuda, cube5):
    """Out-of-range and out-of-order blocks are skipped by the kernel's own
    checks (no access through their indices) and make the dot NaN; the next
    well-formed call is unaffected (the check word is cleared)."""
    import torch

    s = cube5
    rows, col, val = _bcoo(solver, s, cuda)
    lib = solver.lib
    x = to_dev(np.random.default_rng(2).standard_normal(3 * s.n_verts), cuda)
    for bad in ("column", "order"):
        r, c = rows.copy(), col.copy()
        if bad == "column":
            c[len(c) // 2] = s.n_verts + 5
        else:
            r[len(r) // 2], r[len(r) // 2 + 40] = r[len(r) // 2 + 40], r[len(r) // 2]
        y = torch.zeros_like(x)
        dot = torch.zeros(1, dtype=torch.float64, device=cuda)
        rc = _noalloc(lib, s.n_verts, to_dev(r, cuda), to_dev(c, cuda), to_dev(val, cuda), x, y, dot)
        assert rc == 0
        torch.cuda.synchronize()
        assert np.isnan(float(dot.item())), bad
    y = torch.zeros_like(x)
    dot = torch.zeros(1, dtype=torch.float64, device=cuda)
    assert _noalloc(lib, s.n_verts, to_dev(rows, cuda), to_dev(col, cuda), to_dev(val, cuda), x, y, dot) == 0
    torch.cuda.synchronize()
    assert np.isfinite(float(dot.item()))


def test_noalloc_spmv_rejects_oversized_input(cuda):
    from libuipc_b200._native import load_solve_lib

    lib = load_solve_lib()
    one = C.c_void_p(1)  # never dereferenced: the size check comes first
    rc = lib.b2s_spmv_noalloc(1, MAX_BLOCKS + 1, one, one, one, one, one, None, None)
    assert rc == -1
    assert b"limit" in lib.b2s_last_error(None)
