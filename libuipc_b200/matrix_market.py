"""Matrix Market ingest and export of Newton systems, in the format libuipc's
debug dump writes (src/backends/cuda/utils/matrix_market.h: export_matrix_market
:35-116, export_vector_market :126-158, import_matrix_market :247-366,
import_vector_market :376-450; dump call site
src/backends/cuda/linear_system/global_linear_system.cu:34-70 under the scene
setting ``extras/debug/dump_linear_system``).

A system dumped by a GPU build of the reference (A = its assembled block-upper
BCOO, b, x) is read here into triplets that :meth:`Solver.assemble` takes, so
the same assembled system can be solved by both; a system assembled here is
written in the same format. The parsing and formatting are native
(``csrc/scene/matrix_market.cpp``); block values are 9 doubles column-major,
as in the triplet arrays.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._native import load_scene_lib

_ERRORS = {-1: "I/O error", -2: "not a Matrix Market file of the expected kind", -3: "bad argument"}


def _check(code: int, what: str, path: str) -> None:
    if code != 0:
        raise ValueError(f"{what} {path!r}: {_ERRORS.get(code, code)}")


def export_matrix_market(path: str, n_block_rows: int, rows, cols, vals, one_based: bool = True) -> None:
    """Write the 3x3 blocks (rows[k], cols[k], vals[k] column-major) with all
    9 entries of every block, zeros included, as the reference does."""
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    vals = np.ascontiguousarray(vals, dtype=np.float64).reshape(-1, 9)
    if not (len(rows) == len(cols) == len(vals)):
        raise ValueError("rows, cols and vals differ in length")
    lib = load_scene_lib()
    _check(lib.b2io_write_block_matrix(os.fsencode(path), int(n_block_rows), len(rows), rows.ctypes.data,
                                       cols.ctypes.data, vals.ctypes.data, 1 if one_based else 0),
           "cannot write", path)


def export_vector_market(path: str, x) -> None:
    x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).ravel())
    _check(load_scene_lib().b2io_write_vector(os.fsencode(path), len(x), x.ctypes.data), "cannot write", path)


def import_matrix_market(path: str, one_based: bool = True):
    """Returns (n_block_rows, rows int32[K], cols int32[K], vals float64[K, 9])
    with the blocks ordered by (block row, block column)."""
    lib = load_scene_lib()
    h = C.c_void_p()
    _check(lib.b2io_read_block_matrix(os.fsencode(path), 1 if one_based else 0, C.byref(h)), "cannot read", path)
    try:
        nb, k, ne = C.c_int32(), C.c_int64(), C.c_int64()
        lib.b2io_matrix_size(h, C.byref(nb), C.byref(k), C.byref(ne))
        rows = np.empty(k.value, np.int32)
        cols = np.empty(k.value, np.int32)
        vals = np.empty((k.value, 9), np.float64)
        lib.b2io_matrix_copy(h, rows.ctypes.data, cols.ctypes.data, vals.ctypes.data)
    finally:
        lib.b2io_matrix_free(h)
    return nb.value, rows, cols, vals


def import_vector_market(path: str) -> np.ndarray:
    lib = load_scene_lib()
    n = C.c_int64()
    _check(lib.b2io_read_vector(os.fsencode(path), 0, None, C.byref(n)), "cannot read", path)
    x = np.empty(n.value, np.float64)
    _check(lib.b2io_read_vector(os.fsencode(path), n.value, x.ctypes.data, C.byref(n)), "cannot read", path)
    return x


def export_assembled(solver, path: str, one_based: bool = True) -> None:
    """The solver's assembled block-upper matrix (the reference dumps its
    bcoo_A, the same pattern) as a Matrix Market file."""
    rowptr, col, vals = solver.upper_bsr()
    rows = np.repeat(np.arange(len(rowptr) - 1, dtype=np.int32), np.diff(rowptr))
    export_matrix_market(path, len(rowptr) - 1, rows, col, vals, one_based)


def dump_names(folder: str, frame: int, newton_iter: int) -> tuple[str, str, str]:
    """The reference's file names for A, b and x of one Newton iteration."""
    return tuple(os.path.join(folder, f"{w}.{frame}.{newton_iter}.mtx") for w in ("A", "b", "x"))
