"""Matrix Market dumps through the product path: the GPU-assembled matrix
written in the reference's debug-dump format and read back is the oracle's
convert_sym result bit for bit; a system read from a dump assembles to the
same matrix and solves to the same x (to rounding); the GlobalLinearSystem
mirror writes A, b and x under the reference's file names when its dump
folder is set."""
import os

import numpy as np
import pytest

from conftest import to_dev
from libuipc_b200 import _abi
from libuipc_b200 import matrix_market as mm
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_dump_of_the_gpu_assembly_is_the_oracle_matrix(solver, cuda, cube10, tmp_path):
    s = cube10
    solver.assemble(s.n_verts, to_dev(s.rows, cuda), to_dev(s.cols, cuda), to_dev(s.vals, cuda))
    p = str(tmp_path / "A.mtx")
    mm.export_assembled(solver, p)
    nb, rows, cols, vals = mm.import_matrix_market(p)
    _, orow, ocol, oval = O.OracleMatrix(s.n_verts, s.rows, s.cols, s.vals).bsr()
    assert nb == s.n_verts
    np.testing.assert_array_equal(rows, orow)
    np.testing.assert_array_equal(cols, ocol)
    assert np.array_equal(vals.view(np.int64), oval.view(np.int64))


def test_system_read_from_a_dump_solves_the_same(solver, cuda, cube10, tmp_path):
    import torch

    s = cube10
    b = to_dev(s.b, cuda)
    solver.assemble(s.n_verts, to_dev(s.rows, cuda), to_dev(s.cols, cuda), to_dev(s.vals, cuda))
    solver.precond_assemble(_abi.B2S_PRECOND_JACOBI)
    x1 = torch.zeros_like(b)
    st1 = solver.pcg(b, x1, tol=1e-10, stop_rule=_abi.B2S_STOP_RELRES)
    a_path, b_path = str(tmp_path / "A.1.0.mtx"), str(tmp_path / "b.1.0.mtx")
    mm.export_assembled(solver, a_path)
    mm.export_vector_market(b_path, s.b)
    nb, rows, cols, vals = mm.import_matrix_market(a_path)
    bb = mm.import_vector_market(b_path)
    rp0, c0, v0 = solver.upper_bsr()
    solver.assemble(nb, to_dev(rows, cuda), to_dev(cols, cuda), to_dev(vals, cuda))
    rp1, c1, v1 = solver.upper_bsr()
    assert np.array_equal(rp0, rp1) and np.array_equal(c0, c1) and np.array_equal(v0, v1)
    solver.precond_assemble(_abi.B2S_PRECOND_JACOBI)
    x2 = torch.zeros_like(b)
    st2 = solver.pcg(to_dev(bb, cuda), x2, tol=1e-10, stop_rule=_abi.B2S_STOP_RELRES)
    # the same matrix and b; the SpMV's transposed half is reduced with
    # atomics, so the two solves agree to rounding amplified by the iteration
    # (measured 8e-12 relative at a 1e-10 stop), not bit for bit
    assert abs(st1["iterations_exact"] - st2["iterations_exact"]) <= 5
    assert float(torch.linalg.norm(x1 - x2)) <= 1e-9 * float(torch.linalg.norm(x1))


def test_global_linear_system_dump(solver, cuda, cube10, tmp_path):
    from libuipc_b200.linear_system import B200Jacobi, B200PCG, GlobalLinearSystem, dump_folder_from_config

    s = cube10
    folder = dump_folder_from_config({"extras/debug/dump_linear_system": 1}, str(tmp_path))
    assert dump_folder_from_config({}, str(tmp_path)) is None
    pcg = B200PCG(tol_rate=1e-10, stop_rule=_abi.B2S_STOP_RELRES)
    gls = GlobalLinearSystem(solver, pcg, B200Jacobi(), dump_folder=folder)
    dx = gls.solve(s.n_verts, to_dev(s.rows, cuda), to_dev(s.cols, cuda), to_dev(s.vals, cuda), to_dev(s.b, cuda),
                   frame=3, newton_iter=1)
    a_path, b_path, x_path = mm.dump_names(folder, 3, 1)
    assert all(os.path.exists(p) for p in (a_path, b_path, x_path))
    _, rows, cols, vals = mm.import_matrix_market(a_path)
    _, orow, ocol, oval = O.OracleMatrix(s.n_verts, s.rows, s.cols, s.vals).bsr()
    assert np.array_equal(rows, orow) and np.array_equal(cols, ocol) and np.array_equal(vals, oval)
    assert np.array_equal(mm.import_vector_market(b_path), s.b)
    assert np.array_equal(mm.import_vector_market(x_path), -dx.cpu().numpy())
