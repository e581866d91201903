"""Loading of the in-tree native libraries.

``libb200solve.so`` is the product (CUDA kernels for sm_100a behind a C ABI,
declared in ``include/b200solve.h``); ``libb200scene.so`` is the host-side
synthetic Newton-system generator. Both are built in-tree by
``libuipc_b200/build.py``. There is no fallback: a missing or stale library
raises, so nothing silently runs on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib")
_lock = threading.Lock()
_scene = None
_solve = None

c_int_p = C.POINTER(C.c_int)
c_i32_p = C.POINTER(C.c_int32)
c_i64_p = C.POINTER(C.c_int64)
c_dbl_p = C.POINTER(C.c_double)


def lib_path(name: str) -> str:
    return os.path.join(_LIB_DIR, name)


def _load(name: str) -> C.CDLL:
    path = lib_path(name)
    if not os.path.exists(path):
        raise RuntimeError(
            f"native library {path} is missing; build it with `python -m libuipc_b200.build`"
        )
    return C.CDLL(path, mode=C.RTLD_GLOBAL)


def load_scene_lib() -> C.CDLL:
    global _scene
    with _lock:
        if _scene is not None:
            return _scene
        lib = _load("libb200scene.so")
        vp = C.c_void_p
        lib.b2g_default_config.argtypes = [C.c_void_p]
        lib.b2g_default_config.restype = None
        lib.b2g_generate.argtypes = [C.c_void_p, C.POINTER(vp)]
        lib.b2g_generate.restype = C.c_int
        lib.b2g_generate_state.argtypes = [C.c_void_p, c_dbl_p, c_dbl_p, C.POINTER(vp)]
        lib.b2g_generate_state.restype = C.c_int
        lib.b2g_free.argtypes = [vp]
        lib.b2g_free.restype = None
        lib.b2g_last_error.argtypes = []
        lib.b2g_last_error.restype = C.c_char_p
        for fn in ("b2g_num_verts", "b2g_num_tets", "b2g_num_triplets", "b2g_num_contacts", "b2g_num_adjacency",
                   "b2g_num_bodies"):
            getattr(lib, fn).argtypes = [vp]
            getattr(lib, fn).restype = C.c_int64
        for fn in ("b2g_positions", "b2g_rest_positions", "b2g_triplet_vals", "b2g_gradient"):
            getattr(lib, fn).argtypes = [vp]
            getattr(lib, fn).restype = c_dbl_p
        for fn in ("b2g_tets", "b2g_triplet_rows", "b2g_triplet_cols", "b2g_adjacency_start", "b2g_adjacency_list"):
            getattr(lib, fn).argtypes = [vp]
            getattr(lib, fn).restype = c_i32_p
        dp = C.POINTER(C.c_double)
        lib.b2g_element_bw.argtypes = [vp, vp, C.c_double, C.c_double, C.c_double, C.c_double, vp, vp]
        lib.b2g_element_bw.restype = C.c_double
        lib.b2g_element_dsb.argtypes = [vp, vp, C.c_double, C.c_double, vp, vp]
        lib.b2g_element_dsb.restype = C.c_double
        lib.b2g_element_ortho.argtypes = [vp, C.c_double, C.c_double, vp, vp]
        lib.b2g_element_ortho.restype = C.c_double
        lib.b2g_element_contact.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.c_double, vp, vp]
        lib.b2g_element_contact.restype = C.c_int
        lib.b2g_contact_energy.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.c_double]
        lib.b2g_contact_energy.restype = C.c_double
        lib.b2g_accd.argtypes = [vp, vp, C.c_int, C.c_double, C.c_double, C.c_int, C.c_double,
                                 C.POINTER(C.c_double)]
        lib.b2g_accd.restype = C.c_int
        # Matrix Market I/O (csrc/scene/matrix_market.h)
        i32, i64, pi32, pi64 = C.c_int32, C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_int64)
        lib.b2io_write_block_matrix.argtypes = [C.c_char_p, i32, i64, vp, vp, vp, C.c_int]
        lib.b2io_write_block_matrix.restype = C.c_int
        lib.b2io_write_vector.argtypes = [C.c_char_p, i64, vp]
        lib.b2io_write_vector.restype = C.c_int
        lib.b2io_read_block_matrix.argtypes = [C.c_char_p, C.c_int, C.POINTER(vp)]
        lib.b2io_read_block_matrix.restype = C.c_int
        lib.b2io_matrix_size.argtypes = [vp, pi32, pi64, pi64]
        lib.b2io_matrix_size.restype = C.c_int
        lib.b2io_matrix_copy.argtypes = [vp, vp, vp, vp]
        lib.b2io_matrix_copy.restype = C.c_int
        lib.b2io_matrix_free.argtypes = [vp]
        lib.b2io_matrix_free.restype = None
        lib.b2io_read_vector.argtypes = [C.c_char_p, i64, vp, pi64]
        lib.b2io_read_vector.restype = C.c_int
        _scene = lib
        return lib


def load_solve_lib() -> C.CDLL:
    """Load libb200solve.so and declare every entry point of include/b200solve.h."""
    global _solve
    with _lock:
        if _solve is not None:
            return _solve
        lib = _load("libb200solve.so")
        from ._abi import declare

        declare(lib)
        _solve = lib
        return lib
