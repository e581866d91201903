"""The solve over linear subsystems on the device
(GlobalLinearSystem.solve_subsystems): an affine body (uid 0, first), a tet
cube (uid 1) and a coupling between them, laid out, filled and written into
device arrays, assembled, preconditioned (3x3 Jacobi on the cube, the body's
12x12 block inverse on its rows) and solved to rel-res 1e-10; dx agrees with a
direct solve of the same triplets assembled by the oracle (relative 1e-6) and
every subsystem receives its slice of dx."""
import numpy as np
import pytest

from libuipc_b200 import _abi
from oracle import oracle as O
from test_subsystems_cpu import Body, Coupling, Mesh, _spd

pytestmark = pytest.mark.gpu


def test_subsystems_solve_on_the_device(solver, cuda, cube5):
    import scipy.sparse.linalg as spla

    from libuipc_b200.linear_system import B200Jacobi, B200PCG, GlobalLinearSystem
    from libuipc_b200.subsystems import SubsystemLayout

    s = cube5
    rng = np.random.default_rng(11)
    d = float(np.abs(s.vals[:, [0, 4, 8]]).max())
    body = Body(0, _spd(12, rng, d / 24.0), rng.standard_normal(12) * float(np.abs(s.b).max()), spare=3)
    mesh = Mesh(1, s.n_verts, s.rows, s.cols, s.vals, s.b)
    coup = Coupling(4, body, mesh, [(0, 0, 1e-3 * d * rng.standard_normal((3, 3))),
                                    (2, 7, 1e-3 * d * rng.standard_normal((3, 3)))], n_rl=2)
    lay = SubsystemLayout([mesh, body], [coup])
    pcg = B200PCG(tol_rate=1e-10, stop_rule=_abi.B2S_STOP_RELRES)
    gls = GlobalLinearSystem(solver, pcg, B200Jacobi(abd=(0, 1)))
    dx = gls.solve_subsystems(lay).cpu().numpy()
    assert pcg.last_stats["rel_res"] <= 1e-10
    n, T = lay.total_dof, lay.total_triplets
    rows = np.empty(lay.triplet_capacity, np.int32)
    cols = np.empty(lay.triplet_capacity, np.int32)
    vals = np.empty((lay.triplet_capacity, 9))
    b = np.empty(lay.dof_capacity)
    lay.assemble(rows, cols, vals, b)
    A = O.OracleMatrix(lay.n_block_rows, rows[:T], cols[:T], vals[:T]).to_scipy().tocsc()
    xt = spla.spsolve(A, b[:n])
    assert np.linalg.norm(dx + xt) <= 1e-6 * np.linalg.norm(xt)
    assert np.array_equal(body.dx.cpu().numpy() if hasattr(body.dx, "cpu") else body.dx, dx[:12])
    md = mesh.dx.cpu().numpy() if hasattr(mesh.dx, "cpu") else mesh.dx
    assert np.array_equal(md, dx[12:])
    # a second Newton iteration with more body triplets reuses or grows the buffers
    body.spare = 400
    dx2 = gls.solve_subsystems(lay).cpu().numpy()
    assert np.linalg.norm(dx2 - dx) <= 1e-6 * np.linalg.norm(xt)
