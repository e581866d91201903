"""Python access to the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
the checker; the product never imports it.

Parity status: unpinned for the solve math (see oracle.h): libuipc's CUDA
backend cannot be built here and ships no golden vectors for this path. The
MAS partition step is pinned to the reference's own METIS when
oracle/_ref/libmetis_ref.so exists (compiled from the reference sources).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
_metis = None

ORC_PRECOND_NONE = 0
ORC_PRECOND_JACOBI = 1
ORC_PRECOND_MAS = 2
ORC_STOP_RZ = 0
ORC_STOP_RELRES = 1


class OrcPcgResult(C.Structure):
    _fields_ = [
        ("iterations", C.c_int64),
        ("converged", C.c_int64),
        ("rz0", C.c_double),
        ("rel_res_true", C.c_double),
        ("bypassed", C.c_int64),
    ]


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    path = os.path.join(HERE, "_build", "liboracle.so")
    if not os.path.exists(path):
        from . import build_oracle

        build_oracle.build_oracle_lib()
    L = C.CDLL(path)
    vp, i32, i64, d = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    L.orc_assemble.restype = vp
    L.orc_assemble.argtypes = [i32, i64, vp, vp, vp]
    L.orc_matrix_free.argtypes = [vp]
    L.orc_matrix_nnz.restype = i64
    L.orc_matrix_nnz.argtypes = [vp]
    L.orc_matrix_rows.restype = i32
    L.orc_matrix_rows.argtypes = [vp]
    L.orc_matrix_copy.argtypes = [vp, vp, vp, vp, vp]
    L.orc_spmv.argtypes = [vp, d, vp, d, vp]
    L.orc_mas_create.restype = vp
    L.orc_mas_create.argtypes = [i32, vp, vp, i32, vp, vp]
    L.orc_mas_free.argtypes = [vp]
    L.orc_mas_level_num.restype = i32
    L.orc_mas_level_num.argtypes = [vp]
    L.orc_mas_total_nodes.restype = i32
    L.orc_mas_total_nodes.argtypes = [vp]
    L.orc_mas_levels.argtypes = [vp, vp, vp]
    L.orc_mas_hierarchy.argtypes = [vp, vp, vp]
    L.orc_mas_assemble.restype = C.c_int
    L.orc_mas_assemble.argtypes = [vp, vp, i32, C.c_int]
    L.orc_mas_clusters.argtypes = [vp, vp, vp]
    L.orc_mas_apply.argtypes = [vp, vp, vp]
    L.orc_mas_set_inverses.argtypes = [vp, vp]
    L.orc_mas_quantize.argtypes = [vp, C.c_int]
    L.orc_pcg.restype = C.c_int
    L.orc_pcg.argtypes = [vp, C.c_int, vp, i32, vp, vp, d, C.c_int, C.c_int, i64, C.c_int, C.POINTER(OrcPcgResult)]
    L.orc_pcg_abd.restype = C.c_int
    L.orc_pcg_abd.argtypes = [vp, C.c_int, vp, i32, i32, i32, vp, vp, d, C.c_int, C.c_int, i64, C.c_int,
                              C.POINTER(OrcPcgResult)]
    L.orc_cg_truth.restype = C.c_int
    L.orc_cg_truth.argtypes = [vp, vp, vp, d, i64, C.c_int, C.POINTER(C.c_int64)]
    _lib = L
    return L


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class OracleMatrix:
    """convert_sym + BSR offsets restated on the CPU (FP64, source-order sums)."""

    def __init__(self, nb: int, rows: np.ndarray, cols: np.ndarray, vals: np.ndarray):
        L = lib()
        self._rows = np.ascontiguousarray(rows, dtype=np.int32)
        self._cols = np.ascontiguousarray(cols, dtype=np.int32)
        self._vals = np.ascontiguousarray(vals, dtype=np.float64).reshape(-1, 9)
        self.h = L.orc_assemble(int(nb), int(self._rows.size), _p(self._rows), _p(self._cols), _p(self._vals))
        self.nb = int(nb)
        self.nnz = int(L.orc_matrix_nnz(self.h))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_matrix_free(self.h)
            self.h = None

    def bsr(self):
        rowptr = np.zeros(self.nb + 1, np.int32)
        rows = np.zeros(self.nnz, np.int32)
        cols = np.zeros(self.nnz, np.int32)
        vals = np.zeros((self.nnz, 9), np.float64)
        lib().orc_matrix_copy(self.h, _p(rowptr), _p(rows), _p(cols), _p(vals))
        return rowptr, rows, cols, vals

    def spmv(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(3 * self.nb, np.float64)
        lib().orc_spmv(self.h, 1.0, _p(x), 0.0, _p(y))
        return y

    def to_scipy(self):
        import scipy.sparse as sp

        rowptr, rows, cols, vals = self.bsr()
        blocks = vals.reshape(-1, 3, 3).transpose(0, 2, 1)  # column-major -> [k, p, q]
        ii, jj, vv = [], [], []
        p, q = np.meshgrid(np.arange(3), np.arange(3), indexing="ij")
        for k_rows, k_cols, tp in ((rows, cols, False), (cols, rows, True)):
            sel = np.ones(rows.size, bool) if not tp else (rows != cols)
            b = blocks[sel]
            if tp:
                b = b.transpose(0, 2, 1)
            ii.append((3 * k_rows[sel])[:, None, None] + p[None])
            jj.append((3 * k_cols[sel])[:, None, None] + q[None])
            vv.append(b)
        I = np.concatenate([a.ravel() for a in ii])
        J = np.concatenate([a.ravel() for a in jj])
        V = np.concatenate([a.ravel() for a in vv])
        return sp.csr_matrix((V, (I, J)), shape=(3 * self.nb, 3 * self.nb))


class OracleMAS:
    """MAS hierarchy / Galerkin / inversion / apply restated on the CPU."""

    def __init__(self, vn: int, adj_start, adj_list, p2r, r2p):
        L = lib()
        self._a = [np.ascontiguousarray(a, dtype=np.int32) for a in (adj_start, adj_list, p2r, r2p)]
        self.vn = int(vn)
        self.N = int(self._a[2].size)
        self.h = L.orc_mas_create(self.vn, _p(self._a[0]), _p(self._a[1]), self.N, _p(self._a[2]), _p(self._a[3]))
        self.L = int(L.orc_mas_level_num(self.h))
        self.total = int(L.orc_mas_total_nodes(self.h))
        self.clusters = self.total // 16

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_mas_free(self.h)
            self.h = None

    def levels(self):
        b = np.zeros(self.L + 1, np.int32)
        c = np.zeros(self.L + 1, np.int32)
        lib().orc_mas_levels(self.h, _p(b), _p(c))
        return b, c

    def coarse_table(self):
        ct = np.zeros(self.vn * max(self.L - 1, 1), np.int32)
        lib().orc_mas_hierarchy(self.h, None, _p(ct))
        return ct.reshape(self.vn, max(self.L - 1, 1))[:, : self.L - 1]

    def assemble(self, A: OracleMatrix, offset_blocks: int = 0, invert_mode: int = 0):
        lib().orc_mas_assemble(self.h, A.h, int(offset_blocks), int(invert_mode))

    def clusters_arrays(self):
        hess = np.zeros((self.clusters, 136, 9), np.float64)
        inv = np.zeros((self.clusters, 136, 9), np.float32)
        lib().orc_mas_clusters(self.h, _p(hess), _p(inv))
        return hess, inv

    def set_inverses(self, inv: np.ndarray):
        """Use these cluster inverses (float32 [clusters, 136, 9]) instead of
        the oracle's own, e.g. the device's, to compare applies entry for entry."""
        inv = np.ascontiguousarray(inv, dtype=np.float32)
        assert inv.size == self.clusters * 136 * 9
        lib().orc_mas_set_inverses(self.h, _p(inv))

    def quantize(self, mode: int):
        """0 = FP32 inverses, 1 = BF16, 2 = BF16 of the diagonal-scaled inverse."""
        lib().orc_mas_quantize(self.h, int(mode))

    def apply(self, r: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros(3 * self.vn, np.float64)
        lib().orc_mas_apply(self.h, _p(r), _p(z))
        return z


def pcg(A: OracleMatrix, b, precond=ORC_PRECOND_JACOBI, mas: OracleMAS | None = None, mas_offset=0, tol=1e-4,
        stop_rule=ORC_STOP_RZ, check_interval=1, max_iter=0, threads=1, abd=(0, 0)):
    """PCG as the reference runs it; ``abd = (block_offset, n_bodies)`` adds
    the affine bodies' 12x12 block Jacobi on their block rows."""
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    res = OrcPcgResult()
    mi = max_iter if max_iter > 0 else 2 * b.size
    lib().orc_pcg_abd(A.h, precond, mas.h if mas is not None else None, int(mas_offset), int(abd[0]), int(abd[1]),
                      _p(b), _p(x), float(tol), int(stop_rule), int(check_interval), int(mi), int(threads),
                      C.byref(res))
    return x, {k: getattr(res, k) for k, _ in OrcPcgResult._fields_}


def abd_block_jacobi(A_scipy, block_offset: int, n_bodies: int, r: np.ndarray) -> np.ndarray:
    """ABDDiagPreconditioner (src/backends/cuda/affine_body/abd_diag_preconditioner.cu:15-125):
    on block rows [block_offset, block_offset + 4 n_bodies), z_b = H_b^-1 r_b with H_b the
    full 12x12 diagonal block of body b (the symmetric matrix A = U + U^T - diag U), FP64;
    returns z on that range only (length 12 n_bodies)."""
    z = np.zeros(12 * n_bodies)
    for b in range(n_bodies):
        lo = 3 * (block_offset + 4 * b)
        H = A_scipy[lo:lo + 12, lo:lo + 12].toarray()
        z[12 * b:12 * b + 12] = np.linalg.solve(H, r[lo:lo + 12])
    return z


def cg_truth(A: OracleMatrix, b, tol=1e-13, max_iter=0, threads=1):
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    it = C.c_int64(0)
    rc = lib().orc_cg_truth(A.h, _p(b), _p(x), float(tol), int(max_iter or 20 * b.size), int(threads), C.byref(it))
    return x, int(it.value), rc


# ---------------------------------------------------------------------------
# partitions: the reference's METIS (compiled from its own sources)
# ---------------------------------------------------------------------------
def metis_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libmetis_ref.so"))


def _metis_lib():
    global _metis
    if _metis is None:
        _metis = C.CDLL(os.path.join(HERE, "_ref", "libmetis_ref.so"))
        _metis.METIS_SetDefaultOptions.argtypes = [C.c_void_p]
        _metis.METIS_PartGraphKway.argtypes = [C.c_void_p] * 13
        _metis.METIS_PartGraphKway.restype = C.c_int
    return _metis


def metis_mesh_partition(adj_start, adj_list, part_max_size: int = 16) -> np.ndarray:
    """geometry::mesh_partition (src/geometry/mesh_partition.cpp:77-231):
    METIS k-way with seed 0, shrinking the block size until every part holds
    at most part_max_size vertices; sequential fallback."""
    M = _metis_lib()
    n = int(len(adj_start) - 1)
    xadj = np.ascontiguousarray(adj_start, dtype=np.int32)
    adjncy = np.ascontiguousarray(adj_list, dtype=np.int32)
    if adjncy.size == 0:
        return (np.arange(n) // part_max_size).astype(np.int32)
    block = part_max_size
    nparts = 1 + (n - 1) // block
    if nparts <= 1:
        raise ValueError("single-part meshes use connected-component labelling")
    result = np.zeros(n, np.int32)
    ok = False
    while nparts >= 2 and block >= 1:
        opts = np.zeros(40, np.int32)
        M.METIS_SetDefaultOptions(_p(opts))
        opts[9] = 0  # METIS_OPTION_SEED
        nv = np.array([n], np.int32)
        ncon = np.array([1], np.int32)
        npart = np.array([nparts], np.int32)
        cut = np.array([0], np.int32)
        ret = M.METIS_PartGraphKway(_p(nv), _p(ncon), _p(xadj), _p(adjncy), None, None, None, _p(npart), None, None,
                                    _p(opts), _p(cut), _p(result))
        if ret != 1:  # METIS_OK
            break
        if np.bincount(result, minlength=nparts).max() <= part_max_size:
            ok = True
            break
        if block == 1:
            break
        block -= 1
        nparts = 1 + (n - 1) // block
    if not ok:
        result = (np.arange(n) // part_max_size).astype(np.int32)
    return result


# ---------------------------------------------------------------------------
# the RCB partition and the padded maps, restated in numpy (the host arm of
# the benchmark partitions with these, so it loads no product library)
# ---------------------------------------------------------------------------
def rcb_partition(positions: np.ndarray, max_part: int = 16) -> np.ndarray:
    """Recursive coordinate bisection into parts of at most ``max_part``
    vertices, as libb200solve's b2s_partition_rcb computes it: split the
    longest bounding-box axis, the left part holding half the parts' worth of
    vertices (whole parts), vertices ordered by (coordinate, index); parts
    numbered depth-first, left first."""
    pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
    n = pos.shape[0]
    out = np.zeros(n, np.int32)
    if n == 0:
        return out
    stack = [np.arange(n, dtype=np.int64)]
    part = 0
    while stack:
        idx = stack.pop()
        m = idx.size
        if m <= max_part:
            out[idx] = part
            part += 1
            continue
        p = pos[idx]
        ext = p.max(axis=0) - p.min(axis=0)
        axis = 0
        for a in (1, 2):
            if ext[a] > ext[axis]:
                axis = a
        parts_total = (m + max_part - 1) // max_part
        left = ((parts_total + 1) // 2) * max_part
        if left >= m:
            left = m - 1
        order = np.lexsort((idx, p[:, axis]))  # by coordinate, then vertex index
        stack.append(idx[order[left:]])  # right processed after left
        stack.append(idx[order[:left]])
    return out


def partition_maps(part_ids: np.ndarray, max_part: int = 16):
    """FEMMASPreconditioner::do_init step 4 (fem_mas_preconditioner.cu:285-330):
    vertices grouped by part id (parts in id order, vertices ascending), each
    part padded to a multiple of 16 slots; returns (part_to_real, real_to_part)."""
    pid = np.ascontiguousarray(part_ids, dtype=np.int32)
    n = pid.size
    valid = pid >= 0
    n_parts = int(pid.max()) + 1 if valid.any() else 0
    count = np.bincount(pid[valid], minlength=n_parts)
    if count.size and count.max() > max_part:
        raise ValueError("a part holds more than max_part vertices")
    padded = (count + 15) // 16 * 16
    start = np.concatenate([[0], np.cumsum(padded)[:-1]]).astype(np.int64)
    p2r = np.full(int(padded.sum()), -1, np.int32)
    r2p = np.full(n, -1, np.int32)
    order = np.flatnonzero(valid)
    order = order[np.argsort(pid[order], kind="stable")]  # by part, vertices ascending
    rank = np.arange(order.size) - np.repeat(np.concatenate([[0], np.cumsum(count)[:-1]]), count)
    slot = start[pid[order]] + rank
    p2r[slot] = order
    r2p[order] = slot
    return p2r, r2p
