"""CPU tests of the oracle (the checker) against independent computations."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from oracle import oracle as O


def _numpy_assembly(s):
    keep = (s.rows >= 0) & (s.rows <= s.cols)
    key = s.rows[keep].astype(np.int64) * s.n_verts + s.cols[keep]
    uk, inv = np.unique(key, return_inverse=True)
    sums = np.zeros((uk.size, 9))
    np.add.at(sums, inv, s.vals[keep])  # sequential in source order
    return uk, sums


def test_assembly_matches_numpy_bit_exact(cube10):
    A = O.OracleMatrix(cube10.n_verts, cube10.rows, cube10.cols, cube10.vals)
    uk, sums = _numpy_assembly(cube10)
    rowptr, rows, cols, vals = A.bsr()
    assert A.nnz == 9261  # verts + edges of a 10^3 Kuhn grid
    assert np.array_equal(rows.astype(np.int64) * cube10.n_verts + cols, uk)
    assert np.array_equal(vals, sums)
    assert rowptr[0] == 0 and rowptr[-1] == A.nnz and np.all(np.diff(rowptr) >= 0)
    assert np.array_equal(np.repeat(np.arange(cube10.n_verts), np.diff(rowptr)), rows)


def test_assembly_filters_invalid_and_lower():
    rows = np.array([0, 1, 2, -1, 1, 0, 1], np.int32)
    cols = np.array([0, 0, 2, 2, 2, 0, 2], np.int32)
    vals = np.arange(7 * 9, dtype=np.float64).reshape(7, 9)
    A = O.OracleMatrix(3, rows, cols, vals)
    rowptr, r, c, v = A.bsr()
    assert list(r) == [0, 1, 2] and list(c) == [0, 2, 2]
    assert np.array_equal(v[0], vals[0] + vals[5])
    assert np.array_equal(v[1], vals[4] + vals[6])
    assert list(rowptr) == [0, 1, 2, 3]


def test_empty_assembly():
    A = O.OracleMatrix(4, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros((0, 9)))
    rowptr, r, c, v = A.bsr()
    assert A.nnz == 0 and list(rowptr) == [0] * 5


def test_spmv_matches_scipy(cube10):
    A = O.OracleMatrix(cube10.n_verts, cube10.rows, cube10.cols, cube10.vals)
    S = A.to_scipy()
    assert abs(S - S.T).max() == 0.0
    x = np.random.default_rng(0).standard_normal(3 * cube10.n_verts)
    y = A.spmv(x)
    ref = S @ x
    assert np.abs(y - ref).max() <= 1e-14 * np.abs(ref).max()


def test_truth_solve_matches_direct(cube10):
    A = O.OracleMatrix(cube10.n_verts, cube10.rows, cube10.cols, cube10.vals)
    xt = spla.spsolve(A.to_scipy().tocsc(), cube10.b)
    x, it, rc = O.cg_truth(A, cube10.b)
    assert rc == 0
    assert np.linalg.norm(x - xt) <= 1e-10 * np.linalg.norm(xt)


@pytest.mark.parametrize("pre", [O.ORC_PRECOND_NONE, O.ORC_PRECOND_JACOBI])
def test_pcg_reaches_tolerance(cube10, pre):
    A = O.OracleMatrix(cube10.n_verts, cube10.rows, cube10.cols, cube10.vals)
    x, info = O.pcg(A, cube10.b, precond=pre, tol=1e-6, stop_rule=O.ORC_STOP_RELRES)
    assert info["converged"] == 1
    assert info["rel_res_true"] <= 1e-6 * 1.01


def _mas(s, A, part_ids, invert_mode=0):
    from libuipc_b200.linear_system import partition_maps

    p2r, r2p = partition_maps(part_ids)
    M = O.OracleMAS(s.n_verts, s.adj_start, s.adj_list, p2r, r2p)
    M.assemble(A, 0, invert_mode)
    return M


def test_mas_operator_spd_and_fewer_iterations(cube10):
    """MAS is a symmetric positive definite operator and needs fewer PCG
    iterations than 3x3 block Jacobi (the reference's own check,
    apps/tests/sim_case/59_fem_mas_vs_diag_benchmark.cpp:189-191)."""
    from libuipc_b200.linear_system import partition_rcb

    A = O.OracleMatrix(cube10.n_verts, cube10.rows, cube10.cols, cube10.vals)
    M = _mas(cube10, A, partition_rcb(cube10.positions))
    rng = np.random.default_rng(1)
    r1, r2 = rng.standard_normal((2, 3 * cube10.n_verts))
    z1, z2 = M.apply(r1), M.apply(r2)
    assert abs(r2 @ z1 - r1 @ z2) <= 1e-5 * abs(r1 @ z2)
    assert r1 @ z1 > 0 and r2 @ z2 > 0
    _, im = O.pcg(A, cube10.b, precond=O.ORC_PRECOND_MAS, mas=M, tol=1e-4, stop_rule=O.ORC_STOP_RELRES)
    _, ij = O.pcg(A, cube10.b, precond=O.ORC_PRECOND_JACOBI, tol=1e-4, stop_rule=O.ORC_STOP_RELRES)
    assert im["converged"] and ij["converged"]
    assert im["iterations"] < ij["iterations"]


def test_mas_single_bank_is_exact_inverse():
    """A 12-vertex system partitioned into one bank: MAS level 0 is the exact
    inverse (every coarse level adds the Galerkin correction of one node)."""
    from libuipc_b200 import scene
    from libuipc_b200.linear_system import partition_maps

    s = scene.generate(scene=1, cells_x=1, cells_y=1, cells_z=2, seed=4)
    A = O.OracleMatrix(s.n_verts, s.rows, s.cols, s.vals)
    assert s.n_verts == 12
    p2r, r2p = partition_maps(np.zeros(s.n_verts, np.int32))
    M = O.OracleMAS(s.n_verts, s.adj_start, s.adj_list, p2r, r2p)
    M.assemble(A, 0, 1)
    hess, inv = M.clusters_arrays()
    # level-0 cluster matrix equals the assembled matrix
    S = A.to_scipy().toarray()
    H = np.zeros((48, 48))
    for rn in range(16):
        for cn in range(rn, 16):
            si = 16 * rn - rn * (rn + 1) // 2 + cn
            B = hess[0, si].reshape(3, 3).T
            H[3 * rn:3 * rn + 3, 3 * cn:3 * cn + 3] = B
            H[3 * cn:3 * cn + 3, 3 * rn:3 * rn + 3] = B.T
    assert np.allclose(H[:36, :36], S, rtol=0, atol=1e-14 * np.abs(S).max())
    r = np.random.default_rng(2).standard_normal(36)
    z = M.apply(r)
    z0 = np.linalg.solve(S, r)
    # z = z0 + coarse corrections (one node per coarse level)
    assert np.isfinite(z).all() and (r @ z) > (r @ z0) * 0.999


def test_sweep_inverse_matches_numpy(cube10):
    from libuipc_b200.linear_system import partition_rcb

    A = O.OracleMatrix(cube10.n_verts, cube10.rows, cube10.cols, cube10.vals)
    M = _mas(cube10, A, partition_rcb(cube10.positions), invert_mode=0)
    hess, inv = M.clusters_arrays()
    for c in (0, 7, 40):
        H = np.zeros((48, 48))
        Iv = np.zeros((48, 48))
        for rn in range(16):
            for cn in range(rn, 16):
                si = 16 * rn - rn * (rn + 1) // 2 + cn
                B = hess[c, si].reshape(3, 3).T
                H[3 * rn:3 * rn + 3, 3 * cn:3 * cn + 3] = B
                H[3 * cn:3 * cn + 3, 3 * rn:3 * rn + 3] = B.T
                Bi = inv[c, si].reshape(3, 3).T.astype(np.float64)
                Iv[3 * rn:3 * rn + 3, 3 * cn:3 * cn + 3] = Bi
                Iv[3 * cn:3 * cn + 3, 3 * rn:3 * rn + 3] = Bi.T
        d = np.diag(H).copy()
        H[np.arange(48), np.arange(48)] = np.where(d == 0, 1.0, d)
        ref = np.linalg.inv(H)
        assert np.abs(Iv - ref).max() <= 2e-4 * np.abs(ref).max()


def test_metis_partition_pinned_to_reference(cube10):
    """The reference's own METIS (compiled from its sources) yields parts of at
    most 16 vertices covering every vertex."""
    if not O.metis_available():
        pytest.skip("reference METIS not compiled (reference tree absent)")
    pid = O.metis_mesh_partition(cube10.adj_start, cube10.adj_list)
    assert pid.min() == 0 and np.bincount(pid).max() <= 16 and np.bincount(pid).min() >= 1


def test_numpy_rcb_and_maps_equal_the_library(cube10, stack_small):
    """The host arm's numpy RCB and padded maps give the library's partition."""
    from libuipc_b200.linear_system import partition_maps, partition_rcb

    for s in (cube10, stack_small):
        pid = O.rcb_partition(s.positions)
        assert np.array_equal(pid, partition_rcb(s.positions))
        p2r, r2p = O.partition_maps(pid)
        lp2r, lr2p = partition_maps(pid)
        assert np.array_equal(p2r, lp2r) and np.array_equal(r2p, lr2p)
    pid = np.array([0, -1, 0, 1, -1], np.int32)
    p2r, r2p = O.partition_maps(pid)
    assert list(r2p) == [0, -1, 1, 16, -1] and p2r.size == 32
