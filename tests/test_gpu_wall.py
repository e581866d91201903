"""The full-scale scene kind at a reduced size (a 2 x 2 grid of 6^3-cell tet
cubes, a 40 x 40 cloth resting on them, 2 x 2 affine bodies on the cloth):
3x3 tet and cloth blocks, 12x12 body blocks, point-triangle cloth-cube and
12x3 cloth-body couplings in one system. Assembly against the oracle (bit
exact), PCG with MAS on the FEM range and the 12x12 block Jacobi on the bodies
against a direct solve, FP64 and mixed."""
import numpy as np
import pytest

from conftest import to_dev
from libuipc_b200 import _abi
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def wall_small():
    from libuipc_b200 import scene

    return scene.cube_wall(cells=6, side=2, cloth_n=40, bodies_x=2, bodies_z=2, seed=5)


def test_wall_system_has_every_block_kind(wall_small):
    s = wall_small
    assert s.n_bodies == 4 and s.n_contacts > 0
    off = 4 * s.n_bodies
    cubes = 4 * 7 ** 3
    r, c = s.rows, s.cols
    cloth_cube = np.any((r >= off) & (r < off + cubes) & (c >= off + cubes))
    cloth_body = np.any((r < off) & (c >= off + cubes))
    assert cloth_cube and cloth_body


def test_wall_assembly_bit_exact(solver, cuda, wall_small):
    s = wall_small
    solver.assemble(s.n_verts, to_dev(s.rows, cuda), to_dev(s.cols, cuda), to_dev(s.vals, cuda))
    rp, col, val = solver.upper_bsr()
    orp, _, ocol, oval = O.OracleMatrix(s.n_verts, s.rows, s.cols, s.vals).bsr()
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol) and np.array_equal(val, oval)


@pytest.mark.parametrize("precision", [_abi.B2S_PRECISION_FP64, _abi.B2S_PRECISION_MIXED])
def test_wall_pcg_mas_plus_bodies(solver, cuda, wall_small, precision):
    import scipy.sparse.linalg as spla
    import torch

    from libuipc_b200.linear_system import partition_maps, partition_rcb

    s = wall_small
    off = 4 * s.n_bodies
    a0 = s.adj_start[off]
    adj_start = (s.adj_start[off:] - a0).astype(np.int32)
    adj_list = (s.adj_list[a0:] - off).astype(np.int32)
    p2r, r2p = partition_maps(partition_rcb(s.positions[off:]))
    solver.assemble(s.n_verts, to_dev(s.rows, cuda), to_dev(s.cols, cuda), to_dev(s.vals, cuda))
    solver.abd_init(0, s.n_bodies)
    solver.mas_init(off, s.n_verts - off, adj_start, adj_list, p2r, r2p)
    solver.precond_assemble(_abi.B2S_PRECOND_MAS)
    b = to_dev(s.b, cuda)
    x = torch.zeros_like(b)
    st = solver.pcg(b, x, tol=1e-9, stop_rule=_abi.B2S_STOP_RELRES, precision=precision, replace_every=50)
    assert st["converged"] == 1 and st["rel_res"] <= 1e-9
    A = O.OracleMatrix(s.n_verts, s.rows, s.cols, s.vals).to_scipy().tocsc()
    xt = spla.spsolve(A, s.b)
    assert np.linalg.norm(x.cpu().numpy() - xt) <= 1e-5 * np.linalg.norm(xt)
