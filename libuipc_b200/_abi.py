"""ctypes declarations of include/b200solve.h (kept in the header's order)."""
from __future__ import annotations

import ctypes as C

B2S_OK = 0
B2S_ERR_ARGUMENT = -1
B2S_ERR_CUDA = -2
B2S_ERR_STATE = -3
B2S_ERR_NUMERIC = -4
B2S_ERR_NOT_CONVERGED = -5

B2S_PRECOND_NONE = 0
B2S_PRECOND_JACOBI = 1
B2S_PRECOND_MAS = 2

B2S_INVERT_F32 = 0
B2S_INVERT_F64 = 1
B2S_INVERT_F32_ONLY = 2

B2S_STOP_RZ = 0
B2S_STOP_RELRES = 1

B2S_PRECISION_FP64 = 0
B2S_PRECISION_MIXED = 1


B2S_WS_MODE_ZERO = 0
B2S_WS_MODE_PREV = 1
B2S_WS_MODE_HISTORY = 2
B2S_WS_MODE_LEARNED = 3
B2S_WS_HISTORY = 3
B2S_WS_MAX_HISTORY = 8
B2S_WS_FEATURES = 22
B2S_WS_OUTPUTS = 4


class WsInfo(C.Structure):
    _fields_ = [
        ("mode", C.c_int32),
        ("n_candidates", C.c_int32),
        ("coeff", C.c_double * (1 + 8)),
        ("rel_res0", C.c_double),
        ("rel_res_tried", C.c_double),
        ("rz_ratio", C.c_double),
        ("predict_ms", C.c_double),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["coeff"] = list(self.coeff)[: self.n_candidates]
        return d


class PcgOptions(C.Structure):
    _fields_ = [
        ("tol", C.c_double),
        ("stop_rule", C.c_int32),
        ("check_interval", C.c_int32),
        ("max_iter", C.c_int64),
        ("precision", C.c_int32),
        ("use_graph", C.c_int32),
        ("x0_given", C.c_int32),
        ("replace_every", C.c_int32),
    ]


class PcgStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int64),
        ("iterations_exact", C.c_int64),
        ("converged", C.c_int32),
        ("bypassed", C.c_int32),
        ("rz0", C.c_double),
        ("rel_res", C.c_double),
        ("replacements", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Timers(C.Structure):
    _fields_ = [
        ("assemble_ms", C.c_double),
        ("precond_build_ms", C.c_double),
        ("pcg_ms", C.c_double),
        ("spmv_ms", C.c_double),
        ("spmv_launches", C.c_int64),
        ("precond_apply_ms", C.c_double),
        ("precond_apply_launches", C.c_int64),
        ("kernel_launches", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


vp = C.c_void_p
i32 = C.c_int32
i64 = C.c_int64
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
dp = C.POINTER(C.c_double)
fp = C.POINTER(C.c_float)

# name -> (restype, argtypes); every entry point of include/b200solve.h
SIGNATURES = {
    "b2s_create": (C.c_int, [C.c_int, C.POINTER(vp)]),
    "b2s_destroy": (C.c_int, [vp]),
    "b2s_last_error": (C.c_char_p, [vp]),
    "b2s_set_stream": (C.c_int, [vp, vp]),
    "b2s_version": (C.c_int, []),
    "b2s_assemble": (C.c_int, [vp, i32, i64, vp, vp, vp]),
    "b2s_triplet_buffers": (C.c_int, [vp, i64, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
    "b2s_assemble_owned": (C.c_int, [vp, i32, i64]),
    "b2s_matrix_info": (C.c_int, [vp, i32p, i64p]),
    "b2s_get_upper_bsr": (C.c_int, [vp, vp, vp, vp]),
    "b2s_spmv": (C.c_int, [vp, vp, vp, dp]),
    "b2s_spmv_mixed": (C.c_int, [vp, vp, vp, dp]),
    "b2s_spmv_mixed_timing": (C.c_int, [vp, i32, C.POINTER(C.c_double)]),
    "b2s_mas_init": (C.c_int, [vp, i32, i32, vp, vp, i32, vp, vp]),
    "b2s_mas_info": (C.c_int, [vp, i32p, i32p]),
    "b2s_mas_get_hierarchy": (C.c_int, [vp, vp, vp, vp]),
    "b2s_mas_get_clusters": (C.c_int, [vp, vp, vp]),
    "b2s_mas_stiff_info": (C.c_int, [vp, i32p, vp]),
    "b2s_mas_get_nodes": (C.c_int, [vp, vp, vp]),
    "b2s_partition_rcb": (C.c_int, [i32, vp, i32, vp]),
    "b2s_partition_graph": (C.c_int, [i32, vp, vp, i32, vp]),
    "b2s_partition_maps": (C.c_int, [i32, vp, i32, vp, vp, i32p]),
    "b2s_abd_init": (C.c_int, [vp, i32, i32]),
    "b2s_precond_assemble": (C.c_int, [vp, C.c_int, C.c_int]),
    "b2s_precond_apply": (C.c_int, [vp, vp, vp]),
    "b2s_precond_apply_mixed": (C.c_int, [vp, vp, vp]),
    "b2s_pcg_default_options": (None, [C.POINTER(PcgOptions)]),
    "b2s_pcg": (C.c_int, [vp, vp, vp, C.POINTER(PcgOptions), C.POINTER(PcgStats)]),
    "b2s_set_timing": (C.c_int, [vp, C.c_int]),
    "b2s_get_timers": (C.c_int, [vp, C.POINTER(Timers)]),
    "b2s_reset_timers": (C.c_int, [vp]),
    "b2s_ws_init": (C.c_int, [vp, i32, C.c_uint64]),
    "b2s_ws_add_sample": (C.c_int, [vp, vp, i32, vp, vp]),
    "b2s_ws_num_samples": (C.c_int, [vp, i32p, i64p]),
    "b2s_ws_fit_normalization": (C.c_int, [vp]),
    "b2s_ws_train": (C.c_int, [vp, i32, C.c_double, C.c_uint64, dp]),
    "b2s_ws_loss_grad": (C.c_int, [vp, i32, dp, fp]),
    "b2s_ws_get_params": (C.c_int, [vp, fp, i64p]),
    "b2s_ws_set_params": (C.c_int, [vp, fp, i64]),
    "b2s_ws_put_sample": (C.c_int, [vp, i32, vp, vp, vp, vp, C.c_double]),
    "b2s_ws_get_sample": (C.c_int, [vp, i32, i32p, fp, fp, fp, fp, dp]),
    "b2s_ws_predict": (C.c_int, [vp, i32, vp, i32, vp, vp, C.POINTER(WsInfo)]),
    "b2s_spmv_noalloc": (C.c_int, [i32, i64, vp, vp, vp, vp, vp, vp, vp]),
}


def declare(lib: C.CDLL) -> None:
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)  # raises AttributeError when the symbol is missing
        fn.restype = res
        fn.argtypes = args


def header_symbols(header_path: str, prefix: str = "b2s_") -> list[str]:
    """Function names with `prefix` declared in a C header (for the export check)."""
    import re

    text = open(header_path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(" + prefix + r"[a-z0-9_]+)\s*\(", text)))
