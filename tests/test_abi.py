"""CPU tests of the C-ABI library: it loads, exports every declared entry
point, and its host-only utilities (partitioning) behave."""
import ctypes as C
import os
import subprocess

import numpy as np

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "b200solve.h")
LIB = os.path.join(ROOT, "libuipc_b200", "_lib", "libb200solve.so")


def test_library_exports_every_header_symbol():
    from libuipc_b200 import _abi
    from libuipc_b200._native import load_solve_lib

    lib = load_solve_lib()
    declared = _abi.header_symbols(HEADER)
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in b200solve.h but not exported"
    # the ctypes signature table covers the whole header
    assert sorted(_abi.SIGNATURES) == declared
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l and l.split()[-1].startswith("b2s_")}
    assert set(declared) <= exported


def test_io_library_exports_every_header_symbol():
    """include/b200io.h (Matrix Market I/O) is exported by libb200scene.so."""
    from libuipc_b200 import _abi

    declared = _abi.header_symbols(os.path.join(ROOT, "include", "b200io.h"), prefix="b2io_")
    assert len(declared) == 7
    lib = os.path.join(ROOT, "libuipc_b200", "_lib", "libb200scene.so")
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert set(declared) <= exported


def test_generator_symbols_exported():
    """include/b200gen.h (the GPU Newton-system generator) is exported by libb200solve.so."""
    from libuipc_b200 import _abi

    declared = _abi.header_symbols(os.path.join(ROOT, "include", "b200gen.h"), prefix="b2gen_")
    assert len(declared) == 28
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert set(declared) <= exported


def test_library_is_built_for_sm100a():
    """The build recipe emits sm_100a machine code only (no PTX to JIT, no
    other architecture): a kernel of this library can only run on a B200-class
    device, where the GPU tests launch them."""
    from libuipc_b200 import build

    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert all("sm_" not in f and "compute_" not in f for f in build.NVFLAGS[len(build.ARCH):])


def test_create_without_device_fails_cleanly():
    import torch

    from libuipc_b200._native import load_solve_lib

    if torch.cuda.is_available():
        return
    lib = load_solve_lib()
    h = C.c_void_p()
    rc = lib.b2s_create(0, C.byref(h))
    assert rc != 0 and not h.value
    assert len(lib.b2s_last_error(None)) > 0


def test_null_handle_is_an_argument_error():
    from libuipc_b200._native import load_solve_lib

    lib = load_solve_lib()
    assert lib.b2s_assemble(None, 1, 0, None, None, None) == -1
    assert lib.b2s_pcg(None, None, None, None, None) == -1


def test_rcb_partition_and_maps(cube10):
    from libuipc_b200.linear_system import partition_maps, partition_rcb

    pid = partition_rcb(cube10.positions, 16)
    counts = np.bincount(pid)
    assert counts.max() <= 16 and counts.min() >= 1
    # every part but the last holds exactly 16 vertices
    assert (counts[:-1] == 16).sum() >= len(counts) - 2
    p2r, r2p = partition_maps(pid)
    assert p2r.size % 16 == 0
    valid = p2r >= 0
    assert np.array_equal(np.sort(p2r[valid]), np.arange(cube10.n_verts))
    assert np.all(r2p[p2r[valid]] == np.nonzero(valid)[0])


def test_partition_maps_rejects_oversized_parts():
    from libuipc_b200.linear_system import B200SolveError, partition_maps

    pid = np.zeros(17, np.int32)
    try:
        partition_maps(pid)
    except B200SolveError:
        return
    raise AssertionError("a 17-vertex part was accepted")


def test_partition_maps_unpartitioned_vertices():
    from libuipc_b200.linear_system import partition_maps

    pid = np.array([0, -1, 0, 1, -1], np.int32)
    p2r, r2p = partition_maps(pid)
    assert p2r.size == 32
    assert list(r2p) == [0, -1, 1, 16, -1]


def test_line_search_entry_points_validate_before_the_device():
    """The contact and trajectory-filter constructors reject bad input (vertex
    ids out of range, no pairs, a non-positive dhat or cell) with an argument
    error before touching the device, so they behave the same without a GPU."""
    from libuipc_b200 import _abi
    from libuipc_b200.gpu_scene import _lib

    lib = _lib()
    h = C.c_void_p()
    sv = np.array([0, 1, 2, 3], np.int32)
    se = np.array([[0, 1], [2, 3]], np.int32)
    st = np.array([[0, 1, 2]], np.int32)
    rc = lib.b2gen_trajectory_create(0, 3, 4, sv.ctypes.data, 2, se.ctypes.data, 1, st.ctypes.data, 1e-3, 1e-2,
                                     C.byref(h))
    assert rc == _abi.B2S_ERR_ARGUMENT and b"out of range" in lib.b2gen_trajectory_last_error()
    for dhat, cell in ((0.0, 1e-2), (1e-3, 0.0), (float("nan"), 1e-2)):
        rc = lib.b2gen_trajectory_create(0, 4, 4, sv.ctypes.data, 2, se.ctypes.data, 1, st.ctypes.data, dhat, cell,
                                         C.byref(h))
        assert rc == _abi.B2S_ERR_ARGUMENT
    pairs = np.array([[0, 1, 2, -1]], np.int32)
    ee, eps = np.zeros(1, np.uint8), np.zeros(1)
    rc = lib.b2gen_contacts_create(0, 1, pairs.ctypes.data, ee.ctypes.data, eps.ctypes.data, 1e-3, 1e6, 1e-2,
                                   C.byref(h))
    assert rc == _abi.B2S_ERR_ARGUMENT
    rc = lib.b2gen_contacts_create(0, 0, pairs.ctypes.data, ee.ctypes.data, eps.ctypes.data, 1e-3, 1e6, 1e-2,
                                   C.byref(h))
    assert rc == _abi.B2S_ERR_ARGUMENT
    for f in (lib.b2gen_contacts_energy, ):
        assert f(None, None, None, None) == _abi.B2S_ERR_ARGUMENT
    assert lib.b2gen_contacts_toi(None, None, None, 1.0, None, None) == _abi.B2S_ERR_ARGUMENT
    assert lib.b2gen_trajectory_toi(None, None, None, 1.0, None, None) == _abi.B2S_ERR_ARGUMENT
    assert lib.b2gen_trajectory_detect(None, None, None, 1.0, None, None) == _abi.B2S_ERR_ARGUMENT
