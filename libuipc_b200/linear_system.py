"""Host-side mirror of libuipc's linear-system plug-in interface over the C ABI.

libuipc's CUDA backend solves one Newton step through three sim-system
interfaces (src/backends/cuda/linear_system/):
  * GlobalLinearSystem (global_linear_system.h:28-438): owns the triplets,
    the assembled block matrix, x and b; build_linear_system / solve /
    distribute_solution;
  * IterativeSolver (iterative_solver.h:8-62): do_build, do_solve(SolvingInfo)
    with helpers spmv / spmv_dot / apply_preconditioner;
  * GlobalPreconditioner (global_preconditioner.h:8-26): do_assemble(A),
    do_apply(r -> z).
This module keeps those names and their argument meaning; every call goes to
libb200solve.so (include/b200solve.h). Device memory is held in torch CUDA
tensors; PyTorch is only the allocator here.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._native import load_solve_lib


class B200SolveError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _torch():
    import torch

    return torch


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr()) if t is not None else None


class Solver:
    """RAII wrapper of a b2s_solver handle (one CUDA device)."""

    def __init__(self, device: int = 0):
        self.lib = load_solve_lib()
        h = C.c_void_p()
        rc = self.lib.b2s_create(int(device), C.byref(h))
        if rc != _abi.B2S_OK:
            raise B200SolveError(rc, self.lib.b2s_last_error(None).decode())
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.lib.b2s_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != _abi.B2S_OK:
            raise B200SolveError(rc, self.lib.b2s_last_error(self.h).decode())

    # ---- assembly ----------------------------------------------------------
    def assemble(self, n_block_rows: int, rows, cols, vals) -> None:
        """rows/cols: int32 [T], vals: float64 [T, 9] (column-major blocks),
        device tensors."""
        T = int(rows.numel())
        self._check(self.lib.b2s_assemble(self.h, int(n_block_rows), T, _ptr(rows), _ptr(cols), _ptr(vals)))

    def triplet_buffers(self, n_triplets: int):
        """Device addresses (rows, cols, vals) of solver-owned room for
        n_triplets raw triplets (b2s_triplet_buffers): producers write there
        and :meth:`assemble_owned` assembles in place."""
        r, c, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
        self._check(self.lib.b2s_triplet_buffers(self.h, int(n_triplets), C.byref(r), C.byref(c), C.byref(v)))
        return r.value, c.value, v.value

    def assemble_owned(self, n_block_rows: int, n_triplets: int) -> None:
        self._check(self.lib.b2s_assemble_owned(self.h, int(n_block_rows), int(n_triplets)))

    def matrix_info(self):
        nb = C.c_int32()
        nnz = C.c_int64()
        self._check(self.lib.b2s_matrix_info(self.h, C.byref(nb), C.byref(nnz)))
        return nb.value, nnz.value

    def upper_bsr(self):
        nb, nnz = self.matrix_info()
        rowptr = np.zeros(nb + 1, np.int32)
        col = np.zeros(max(nnz, 1), np.int32)
        vals = np.zeros((max(nnz, 1), 9), np.float64)
        self._check(self.lib.b2s_get_upper_bsr(self.h, rowptr.ctypes.data, col.ctypes.data, vals.ctypes.data))
        return rowptr, col[:nnz], vals[:nnz]

    # ---- SpMV ----------------------------------------------------------------
    def spmv(self, x, y, with_dot: bool = False):
        d = C.c_double(0.0)
        self._check(self.lib.b2s_spmv(self.h, _ptr(x), _ptr(y), C.byref(d) if with_dot else None))
        return d.value if with_dot else None

    def spmv_mixed_timing(self, launches: int = 50) -> float:
        """Average duration [ms] of the FP32 SpMV kernel launched back to back
        on the assembled matrix (b2s_spmv_mixed_timing)."""
        ms = C.c_double()
        self._check(self.lib.b2s_spmv_mixed_timing(self.h, int(launches), C.byref(ms)))
        return float(ms.value)

    def spmv_mixed(self, x32, y32, with_dot: bool = False):
        """y = A x as the mixed-precision PCG computes it (FP32 vectors)."""
        d = C.c_double(0.0)
        self._check(self.lib.b2s_spmv_mixed(self.h, _ptr(x32), _ptr(y32), C.byref(d) if with_dot else None))
        return d.value if with_dot else None

    # ---- MAS ---------------------------------------------------------------------
    def mas_init(self, block_offset: int, vert_num: int, adj_start, adj_list, part_to_real, real_to_part):
        a = [np.ascontiguousarray(v, dtype=np.int32) for v in (adj_start, adj_list, part_to_real, real_to_part)]
        self._check(
            self.lib.b2s_mas_init(self.h, int(block_offset), int(vert_num), a[0].ctypes.data,
                                  a[1].ctypes.data if a[1].size else None, int(a[2].size), a[2].ctypes.data,
                                  a[3].ctypes.data)
        )

    def mas_info(self):
        L = C.c_int32()
        tot = C.c_int32()
        self._check(self.lib.b2s_mas_info(self.h, C.byref(L), C.byref(tot)))
        return L.value, tot.value

    def mas_hierarchy(self, vert_num: int):
        L, _ = self.mas_info()
        b = np.zeros(L + 1, np.int32)
        c = np.zeros(L + 1, np.int32)
        ct = np.zeros(max(vert_num * (L - 1), 1), np.int32)
        self._check(self.lib.b2s_mas_get_hierarchy(self.h, b.ctypes.data, c.ctypes.data, ct.ctypes.data))
        return b, c, ct[: vert_num * (L - 1)].reshape(vert_num, L - 1)

    def mas_clusters(self):
        L, tot = self.mas_info()
        ncl = tot // 16
        hess = np.zeros((ncl, 136, 9), np.float64)
        inv = np.zeros((ncl, 136, 9), np.float32)
        self._check(self.lib.b2s_mas_get_clusters(self.h, hess.ctypes.data, inv.ctypes.data))
        return hess, inv

    def mas_stiff(self):
        """(count, flags uint8 [clusters]) of the clusters the last build
        inverted in FP64."""
        L, tot = self.mas_info()
        flags = np.zeros(max(tot // 16, 1), np.uint8)
        n = C.c_int32(0)
        self._check(self.lib.b2s_mas_stiff_info(self.h, C.byref(n), flags.ctypes.data))
        return int(n.value), flags[: tot // 16]

    def mas_nodes(self):
        """(R, Z) node buffers of the last apply, float32 [total_nodes, 3]."""
        L, tot = self.mas_info()
        R = np.zeros((tot, 3), np.float32)
        Z = np.zeros((tot, 3), np.float32)
        self._check(self.lib.b2s_mas_get_nodes(self.h, R.ctypes.data, Z.ctypes.data))
        return R, Z

    # ---- preconditioner ----------------------------------------------------------
    def abd_init(self, block_offset: int, n_bodies: int):
        """Affine bodies on block rows [block_offset, block_offset + 4 n_bodies):
        12x12 block-Jacobi there (ABDDiagPreconditioner)."""
        self._check(self.lib.b2s_abd_init(self.h, int(block_offset), int(n_bodies)))

    def precond_assemble(self, kind: int, invert_mode: int = _abi.B2S_INVERT_F32):
        self._check(self.lib.b2s_precond_assemble(self.h, int(kind), int(invert_mode)))

    def precond_apply(self, r, z):
        self._check(self.lib.b2s_precond_apply(self.h, _ptr(r), _ptr(z)))

    def precond_apply_mixed(self, r32, z32):
        """Mixed-precision apply (FP32 vectors, BF16 diagonal-scaled MAS inverses)."""
        self._check(self.lib.b2s_precond_apply_mixed(self.h, _ptr(r32), _ptr(z32)))

    # ---- PCG -------------------------------------------------------------------------
    def pcg(self, b, x, tol=1e-3, stop_rule=_abi.B2S_STOP_RZ, check_interval=5, max_iter=0,
            precision=_abi.B2S_PRECISION_FP64, use_graph=True, x0_given=False, replace_every=0) -> dict:
        o = _abi.PcgOptions()
        self.lib.b2s_pcg_default_options(C.byref(o))
        o.tol = float(tol)
        o.stop_rule = int(stop_rule)
        o.check_interval = int(check_interval)
        o.max_iter = int(max_iter)
        o.precision = int(precision)
        o.use_graph = 1 if use_graph else 0
        o.x0_given = 1 if x0_given else 0
        o.replace_every = int(replace_every)
        st = _abi.PcgStats()
        rc = self.lib.b2s_pcg(self.h, _ptr(b), _ptr(x), C.byref(o), C.byref(st))
        self._check(rc)
        return st.as_dict()


    # ---- stage timers --------------------------------------------------------------
    def set_timing(self, enable: bool = True):
        self._check(self.lib.b2s_set_timing(self.h, 1 if enable else 0))

    def timers(self) -> dict:
        t = _abi.Timers()
        self._check(self.lib.b2s_get_timers(self.h, C.byref(t)))
        return t.as_dict()

    def reset_timers(self):
        self._check(self.lib.b2s_reset_timers(self.h))

    def set_stream(self, stream_handle: int | None):
        self._check(self.lib.b2s_set_stream(self.h, C.c_void_p(stream_handle) if stream_handle else None))

    # ---- learned warm start (no counterpart in the reference) ---------------
    @staticmethod
    def _hist(history):
        history = [h for h in (history or []) if h is not None][: _abi.B2S_WS_MAX_HISTORY]
        arr = (C.c_void_p * max(len(history), 1))(*[h.data_ptr() for h in history])
        return len(history), arr

    def ws_init(self, hidden: int = 128, seed: int = 0):
        self._check(self.lib.b2s_ws_init(self.h, int(hidden), int(seed)))

    def ws_add_sample(self, b, x, history=()):
        """Store this system's aggregates with its solved x (device tensors);
        history: the latest earlier solutions, newest first."""
        n, arr = self._hist(history)
        self._check(self.lib.b2s_ws_add_sample(self.h, _ptr(b), n, C.cast(arr, C.c_void_p), _ptr(x)))

    def ws_num_samples(self):
        n = C.c_int32()
        rows = C.c_int64()
        self._check(self.lib.b2s_ws_num_samples(self.h, C.byref(n), C.byref(rows)))
        return int(n.value), int(rows.value)

    def ws_fit_normalization(self):
        self._check(self.lib.b2s_ws_fit_normalization(self.h))

    def ws_train(self, epochs: int, lr: float = 1e-3, seed: int = 0) -> float:
        loss = C.c_double()
        self._check(self.lib.b2s_ws_train(self.h, int(epochs), float(lr), int(seed), C.byref(loss)))
        return float(loss.value)

    def ws_params(self) -> np.ndarray:
        n = C.c_int64()
        self._check(self.lib.b2s_ws_get_params(self.h, None, C.byref(n)))
        out = np.zeros(n.value, np.float32)
        self._check(self.lib.b2s_ws_get_params(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), C.byref(n)))
        return out

    def ws_set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._check(self.lib.b2s_ws_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), int(p.size)))

    def ws_loss_grad(self, index: int):
        n_all = self.ws_params().size - 2 * _abi.B2S_WS_FEATURES
        g = np.zeros(n_all, np.float32)
        loss = C.c_double()
        self._check(self.lib.b2s_ws_loss_grad(self.h, int(index), C.byref(loss),
                                              g.ctypes.data_as(C.POINTER(C.c_float))))
        return float(loss.value), g

    def ws_put_sample(self, feat, H, q, c0, norm: float):
        """Append a stored sample from host arrays (the layout ws_sample returns)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (feat, H, q, c0)]
        rows = arrs[3].size
        self._check(self.lib.b2s_ws_put_sample(self.h, int(rows), *[a.ctypes.data for a in arrs], float(norm)))

    def ws_sample(self, index: int) -> dict:
        rows = C.c_int32()
        fp = C.POINTER(C.c_float)
        self._check(self.lib.b2s_ws_get_sample(self.h, int(index), C.byref(rows), None, None, None, None, None))
        r = rows.value
        F, O = _abi.B2S_WS_FEATURES, _abi.B2S_WS_OUTPUTS
        feat = np.zeros((r, F), np.float32)
        H = np.zeros((r, O * (O + 1) // 2), np.float32)
        q = np.zeros((r, O), np.float32)
        c0 = np.zeros(r, np.float32)
        norm = C.c_double()
        self._check(self.lib.b2s_ws_get_sample(self.h, int(index), C.byref(rows), feat.ctypes.data_as(fp),
                                               H.ctypes.data_as(fp), q.ctypes.data_as(fp), c0.ctypes.data_as(fp),
                                               C.byref(norm)))
        return {"feat": feat, "H": H, "q": q, "c0": c0, "norm": float(norm.value)}

    def ws_predict(self, b, x0, history=(), mode=_abi.B2S_WS_MODE_LEARNED) -> dict:
        """Warm start x0 (device tensor, written) for the current system."""
        n, arr = self._hist(history)
        info = _abi.WsInfo()
        self._check(self.lib.b2s_ws_predict(self.h, int(mode), _ptr(b), n, C.cast(arr, C.c_void_p), _ptr(x0),
                                            C.byref(info)))
        return info.as_dict()


def partition_rcb(positions: np.ndarray, max_part: int = 16) -> np.ndarray:
    lib = load_solve_lib()
    pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(pos.shape[0], np.int32)
    rc = lib.b2s_partition_rcb(int(pos.shape[0]), pos.ctypes.data, int(max_part), out.ctypes.data)
    if rc != 0:
        raise B200SolveError(rc, "b2s_partition_rcb failed")
    return out


def partition_graph(adj_start: np.ndarray, adj_list: np.ndarray, max_part: int = 16) -> np.ndarray:
    """Part id of every vertex from the vertex adjacency alone (the library's
    drop-in for geometry::mesh_partition's METIS k-way call)."""
    lib = load_solve_lib()
    xs = np.ascontiguousarray(adj_start, dtype=np.int32)
    xl = np.ascontiguousarray(adj_list, dtype=np.int32)
    n = xs.size - 1
    out = np.zeros(max(n, 0), np.int32)
    rc = lib.b2s_partition_graph(int(n), xs.ctypes.data, xl.ctypes.data, int(max_part), out.ctypes.data)
    if rc != 0:
        raise B200SolveError(rc, "b2s_partition_graph failed")
    return out


def partition_maps(part_ids: np.ndarray, max_part: int = 16):
    lib = load_solve_lib()
    pid = np.ascontiguousarray(part_ids, dtype=np.int32)
    n = int(pid.size)
    size = C.c_int32()
    r2p = np.zeros(max(n, 1), np.int32)
    rc = lib.b2s_partition_maps(n, pid.ctypes.data, int(max_part), None, r2p.ctypes.data, C.byref(size))
    if rc != 0:
        raise B200SolveError(rc, "b2s_partition_maps failed (part larger than max_part?)")
    p2r = np.zeros(max(size.value, 1), np.int32)
    rc = lib.b2s_partition_maps(n, pid.ctypes.data, int(max_part), p2r.ctypes.data, r2p.ctypes.data, C.byref(size))
    if rc != 0:
        raise B200SolveError(rc, "b2s_partition_maps failed")
    return p2r[: size.value], r2p[:n]


# ---------------------------------------------------------------------------
# libuipc-shaped plug-in classes
# ---------------------------------------------------------------------------
@dataclass
class SolvingInfo:
    """GlobalLinearSystem::SolvingInfo (global_linear_system.h:228-246)."""

    x: object  # DenseVectorView<Float> (device tensor)
    b: object  # CDenseVectorView<Float>
    iter_count: int = 0
    # B200 extension: which solution history a warm start reads (e.g. the
    # Newton iteration index within a time step)
    history_slot: int = 0


# linear_system/* keys of libuipc's scene configuration
# (src/core/core/scene_default_config.cpp:146-175) with their defaults, and the
# B200 extensions (precision, warm start)
SCENE_CONFIG_DEFAULTS = {
    "linear_system/tol_rate": 1e-3,
    "linear_system/solver": "fused_pcg",
    "linear_system/fem_preconditioner": "diag",
    "linear_system/use_cuda_graph": 1,
    "linear_system/check_interval": 5,
    "linear_system/b200/precision": "fp64",
    "linear_system/b200/warm_start": "zero",
}


def linear_system_config(config: dict | None = None) -> dict:
    """The linear_system/* settings with defaults filled in, checked against
    the reference's schema (tol_rate in (0, 1), solver in {fused_pcg,
    linear_pcg}, fem_preconditioner in {diag, mas}, use_cuda_graph in
    {0, 1, 2}, check_interval >= 1); ValueError otherwise."""
    c = dict(SCENE_CONFIG_DEFAULTS)
    for k, v in (config or {}).items():
        if k.startswith("linear_system/"):
            if k not in SCENE_CONFIG_DEFAULTS:
                raise ValueError(f"unknown linear-system option {k!r}")
            c[k] = v
    tol = float(c["linear_system/tol_rate"])
    if not 0.0 < tol < 1.0:
        raise ValueError("linear_system/tol_rate must lie in (0, 1)")
    if c["linear_system/solver"] not in ("fused_pcg", "linear_pcg"):
        raise ValueError("linear_system/solver must be fused_pcg or linear_pcg")
    if c["linear_system/fem_preconditioner"] not in ("diag", "mas"):
        raise ValueError("linear_system/fem_preconditioner must be diag or mas")
    if int(c["linear_system/use_cuda_graph"]) not in (0, 1, 2):
        raise ValueError("linear_system/use_cuda_graph must be 0, 1 or 2")
    if int(c["linear_system/check_interval"]) < 1:
        raise ValueError("linear_system/check_interval must be >= 1")
    if c["linear_system/b200/precision"] not in ("fp64", "mixed"):
        raise ValueError("linear_system/b200/precision must be fp64 or mixed")
    if c["linear_system/b200/warm_start"] not in ("zero", "prev", "history", "learned"):
        raise ValueError("linear_system/b200/warm_start must be zero, prev, history or learned")
    return c


class GlobalPreconditioner:
    """GlobalPreconditioner (global_preconditioner.h:8-26)."""

    def do_assemble(self, system: "GlobalLinearSystem") -> None:
        raise NotImplementedError

    def do_apply(self, system: "GlobalLinearSystem", r, z) -> None:
        raise NotImplementedError


class IterativeSolver:
    """IterativeSolver (iterative_solver.h:8-62)."""

    def do_solve(self, system: "GlobalLinearSystem", info: SolvingInfo) -> None:
        raise NotImplementedError


class B200MAS(GlobalPreconditioner):
    """MAS over the FEM vertex range, 3x3 block Jacobi elsewhere (the role of
    FEMMASPreconditioner + FEMDiagPreconditioner on this path); with ``abd``
    = (block_offset, n_bodies), the affine bodies' 12x12 block Jacobi
    (ABDDiagPreconditioner) on their range."""

    def __init__(self, block_offset, vert_num, adj_start, adj_list, part_to_real, real_to_part,
                 invert_mode=_abi.B2S_INVERT_F32, abd=None):
        self.args = (block_offset, vert_num, adj_start, adj_list, part_to_real, real_to_part)
        self.invert_mode = invert_mode
        self.abd = abd
        self._initialised_for = None

    def do_assemble(self, system):
        if self._initialised_for is not system.solver:
            system.solver.mas_init(*self.args)
            if self.abd:
                system.solver.abd_init(*self.abd)
            self._initialised_for = system.solver
        system.solver.precond_assemble(_abi.B2S_PRECOND_MAS, self.invert_mode)

    def do_apply(self, system, r, z):
        system.solver.precond_apply(r, z)


class B200Jacobi(GlobalPreconditioner):
    """3x3 block Jacobi (FEMDiagPreconditioner); with ``abd``, the affine
    bodies' 12x12 block Jacobi on their range."""

    def __init__(self, abd=None):
        self.abd = abd
        self._initialised_for = None

    def do_assemble(self, system):
        if self.abd and self._initialised_for is not system.solver:
            system.solver.abd_init(*self.abd)
            self._initialised_for = system.solver
        system.solver.precond_assemble(_abi.B2S_PRECOND_JACOBI)

    def do_apply(self, system, r, z):
        system.solver.precond_apply(r, z)


class B200PCG(IterativeSolver):
    """LinearFusedPCG's role (linear_fused_pcg.cu:851-943) on the B200 path.
    B200 extensions: ``precision`` (FP64 or mixed) and ``warm_start`` (zero,
    prev, history or learned): the solver keeps the last solutions of each
    history slot on the device and starts the PCG from the b2s_ws_predict
    start; the FP64-checked start falls back to zero by itself."""

    WARM = {"zero": _abi.B2S_WS_MODE_ZERO, "prev": _abi.B2S_WS_MODE_PREV, "history": _abi.B2S_WS_MODE_HISTORY,
            "learned": _abi.B2S_WS_MODE_LEARNED}

    def __init__(self, tol_rate=1e-3, stop_rule=_abi.B2S_STOP_RZ, check_interval=5,
                 precision=_abi.B2S_PRECISION_FP64, use_graph=True, warm_start: str = "zero"):
        if warm_start not in self.WARM:
            raise ValueError(f"unknown warm start {warm_start!r}")
        self.kw = dict(tol=tol_rate, stop_rule=stop_rule, check_interval=check_interval, precision=precision,
                       use_graph=use_graph)
        self.warm_start = warm_start
        self.history: dict[int, list] = {}
        self.last_stats: dict | None = None
        self.last_warm_start: dict | None = None

    @classmethod
    def from_config(cls, config: dict | None = None) -> "B200PCG":
        """From libuipc's linear_system/* scene settings: tol_rate with the
        reference's |r.z| stop rule, check_interval (1 for linear_pcg, which
        checks every iteration on the host), use_cuda_graph != 0 = graph
        replay; plus the b200/precision and b200/warm_start extensions."""
        c = linear_system_config(config)
        ci = 1 if c["linear_system/solver"] == "linear_pcg" else int(c["linear_system/check_interval"])
        prec = _abi.B2S_PRECISION_MIXED if c["linear_system/b200/precision"] == "mixed" else _abi.B2S_PRECISION_FP64
        return cls(tol_rate=float(c["linear_system/tol_rate"]), stop_rule=_abi.B2S_STOP_RZ, check_interval=ci,
                   precision=prec, use_graph=int(c["linear_system/use_cuda_graph"]) != 0,
                   warm_start=c["linear_system/b200/warm_start"])

    def do_solve(self, system, info: SolvingInfo):
        hist = self.history.setdefault(info.history_slot, [])
        given = False
        if self.warm_start != "zero" and hist:
            self.last_warm_start = system.solver.ws_predict(info.b, info.x, hist, self.WARM[self.warm_start])
            given = True
        self.last_stats = system.solver.pcg(info.b, info.x, x0_given=given, **self.kw)
        info.iter_count = int(self.last_stats["iterations"])
        if self.warm_start != "zero":
            hist.insert(0, info.x.clone())
            del hist[_abi.B2S_WS_MAX_HISTORY:]


class GlobalLinearSystem:
    """GlobalLinearSystem::solve (global_linear_system.cu:85-106): assemble the
    triplets, build the preconditioner, solve A x = b, dx = -x."""

    def __init__(self, solver: Solver, iterative_solver: IterativeSolver,
                 preconditioner: GlobalPreconditioner | None = None, dump_folder: str | None = None):
        """``dump_folder``: when set, every solve writes its assembled A and b
        before, and x after, as Matrix Market files named like the reference's
        debug dump (GlobalLinearSystem::_dump_A_b / _dump_x,
        global_linear_system.cu:44-70, enabled there by the scene setting
        ``extras/debug/dump_linear_system``; see :func:`dump_folder_from_config`)."""
        self.solver = solver
        self.iterative_solver = iterative_solver
        self.preconditioner = preconditioner or B200Jacobi()
        self.dump_folder = dump_folder
        self.last_solve_iterations = 0

    def build_linear_system(self, n_block_rows, rows, cols, vals):
        self.solver.assemble(n_block_rows, rows, cols, vals)
        self.preconditioner.do_assemble(self)

    def solve(self, n_block_rows, rows, cols, vals, b, history_slot: int = 0, frame: int = 0,
              newton_iter: int = 0):
        torch = _torch()
        self.build_linear_system(n_block_rows, rows, cols, vals)
        names = None
        if self.dump_folder:
            from . import matrix_market as mm

            os.makedirs(self.dump_folder, exist_ok=True)
            names = mm.dump_names(self.dump_folder, frame, newton_iter)
            mm.export_assembled(self.solver, names[0])
            mm.export_vector_market(names[1], b.detach().cpu().numpy())
        x = torch.zeros_like(b)
        info = SolvingInfo(x=x, b=b, history_slot=history_slot)
        self.iterative_solver.do_solve(self, info)
        self.last_solve_iterations = info.iter_count
        if names:
            from . import matrix_market as mm

            mm.export_vector_market(names[2], x.detach().cpu().numpy())
        return -x  # distribute_solution: dx = -x

    def solve_subsystems(self, layout, history_slot: int = 0, frame: int = 0, newton_iter: int = 0):
        """The solve over linear subsystems (``libuipc_b200.subsystems``), as
        GlobalLinearSystem::solve runs it (global_linear_system.cu:85-106,
        321-544): extents and offsets, the -1 / 0 fill, each subsystem's writes
        into device arrays kept at the layout's reserved capacity, the solve, and
        the solution x handed to every diagonal subsystem on its range (each
        subsystem negates it into its dx, as the reference's do); returns
        dx = -x."""
        torch = _torch()
        n, T = layout.update()
        dev = torch.device("cuda", self.solver.device)
        bufs = getattr(self, "_sub_bufs", None)
        if bufs is None or bufs[0].numel() < layout.triplet_capacity or bufs[3].numel() < layout.dof_capacity:
            tc, dc = max(layout.triplet_capacity, 1), max(layout.dof_capacity, 1)
            bufs = (torch.empty(tc, dtype=torch.int32, device=dev), torch.empty(tc, dtype=torch.int32, device=dev),
                    torch.empty((tc, 9), dtype=torch.float64, device=dev),
                    torch.empty(dc, dtype=torch.float64, device=dev))
            self._sub_bufs = bufs
        rows, cols, vals, b = bufs
        layout.assemble(rows, cols, vals, b)
        dx = self.solve(layout.n_block_rows, rows[:T], cols[:T], vals[:T], b[:n], history_slot=history_slot,
                        frame=frame, newton_iter=newton_iter)
        layout.distribute(-dx)
        return dx


def dump_folder_from_config(config: dict | None, workspace: str) -> str | None:
    """The folder of the debug dump when the scene setting
    ``extras/debug/dump_linear_system`` is non-zero (GlobalLinearSystem::do_build,
    global_linear_system.cu:34-40), else None."""
    if int((config or {}).get("extras/debug/dump_linear_system", 0)):
        return os.path.join(workspace, "debug")
    return None
