"""GPU parity tests: the CUDA path (through the C ABI) against the oracle.

Tolerances: assembly pattern and sums are bit-exact (integer pattern, FP64
sums in source order on both sides); SpMV is FP64 with atomics on the
transposed half, so 1e-13 relative; the MAS cluster matrices are FP64 sums in
a different association, 1e-12 relative; the FP32 cluster inverses and the
FP32 MAS apply are compared at 1e-4 relative (FP32 rounding of a 48x48
elimination); PCG iterates match the oracle's iteration count within one
check and the solution within 1e-6 relative at a matched tight tolerance.
"""
import numpy as np
import pytest

from conftest import to_dev
from libuipc_b200 import _abi, scene
from libuipc_b200.linear_system import partition_maps, partition_rcb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _upload(s, dev):
    import torch

    rows = to_dev(s.rows, dev)
    cols = to_dev(s.cols, dev)
    vals = to_dev(s.vals, dev)
    b = to_dev(s.b, dev)
    return rows, cols, vals, b


def _assemble(solver, s, dev):
    rows, cols, vals, b = _upload(s, dev)
    solver.assemble(s.n_verts, rows, cols, vals)
    return b


# ---------------------------------------------------------------------------
# assembly
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("which", ["cube10", "cube5", "stack_small"])
def test_assembly_bit_exact(request, solver, cuda, which):
    s = request.getfixturevalue(which)
    _assemble(solver, s, cuda)
    A = O.OracleMatrix(s.n_verts, s.rows, s.cols, s.vals)
    rp, col, val = solver.upper_bsr()
    orp, orow, ocol, oval = A.bsr()
    assert np.array_equal(rp, orp)
    assert np.array_equal(col, ocol)
    assert np.array_equal(val, oval)  # source-order FP64 sums on both sides


def test_assembly_values_only_8_byte_aligned(solver, cuda, cube5):
    """A value array that starts 8 bytes into a 16-byte line (a view one
    double into a buffer) takes the scalar gathers: same sums bit for bit."""
    import torch

    s = cube5
    buf = torch.zeros(s.vals.size + 1, dtype=torch.float64, device=cuda)
    buf[1:] = torch.from_numpy(np.ascontiguousarray(s.vals).ravel()).to(cuda)
    vals = buf[1:]
    assert vals.data_ptr() % 16 == 8
    solver.assemble(s.n_verts, to_dev(s.rows, cuda), to_dev(s.cols, cuda), vals)
    rp, col, val = solver.upper_bsr()
    orp, orow, ocol, oval = O.OracleMatrix(s.n_verts, s.rows, s.cols, s.vals).bsr()
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol) and np.array_equal(val, oval)


def test_assembly_long_rows(solver, cuda):
    """Rows of thousands of pairs (an affine body under a large cloth), with
    duplicates, sorted by the block-per-row kernel: bit-exact."""
    rng = np.random.default_rng(21)
    nb = 3000
    rows = np.concatenate([np.zeros(6000), np.full(300, 7), rng.integers(0, nb, 4000), np.full(5000, 2999)])
    cols = np.concatenate([rng.integers(0, nb, 6000), rng.integers(7, nb, 300), rng.integers(0, nb, 4000),
                           np.full(5000, 2999)])
    rows, cols = rows.astype(np.int32), cols.astype(np.int32)
    rows[rng.random(rows.size) < 0.01] = -1  # unwritten slots
    vals = rng.standard_normal((rows.size, 9))
    solver.assemble(nb, to_dev(rows, cuda), to_dev(cols, cuda), to_dev(vals, cuda))
    rp, col, val = solver.upper_bsr()
    orp, _, ocol, oval = O.OracleMatrix(nb, rows, cols, vals).bsr()
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol) and np.array_equal(val, oval)


def test_assembly_edge_cases(solver, cuda):
    import torch

    # lower-triangle and unwritten (-1) slots dropped, duplicates summed, an
    # empty row, a row with many duplicates
    rng = np.random.default_rng(7)
    nb = 6
    rows = [0, 1, 2, -1, 1, 0, 1, 5, 5, 3]
    cols = [0, 0, 2, 2, 2, 0, 2, 5, 5, 5]
    rows += [4] * 300
    cols += list(rng.integers(4, 6, 300))
    rows = np.array(rows, np.int32)
    cols = np.array(cols, np.int32)
    vals = rng.standard_normal((rows.size, 9))
    solver.assemble(nb, to_dev(rows, cuda), to_dev(cols, cuda), to_dev(vals, cuda))
    rp, col, val = solver.upper_bsr()
    orp, _, ocol, oval = O.OracleMatrix(nb, rows, cols, vals).bsr()
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol) and np.array_equal(val, oval)
    # empty input
    e = torch.zeros(0, dtype=torch.int32, device=cuda)
    solver.assemble(3, e, e, torch.zeros((0, 9), dtype=torch.float64, device=cuda))
    rp, col, val = solver.upper_bsr()
    assert list(rp) == [0, 0, 0, 0] and col.size == 0


def test_assembly_rejects_out_of_range_column(solver, cuda):
    from libuipc_b200.linear_system import B200SolveError

    rows = np.array([0, 1], np.int32)
    cols = np.array([0, 7], np.int32)
    vals = np.ones((2, 9))
    with pytest.raises(B200SolveError) as ei:
        solver.assemble(3, to_dev(rows, cuda), to_dev(cols, cuda), to_dev(vals, cuda))
    assert ei.value.code == _abi.B2S_ERR_ARGUMENT


# ---------------------------------------------------------------------------
# SpMV
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("which", ["cube10", "stack_small"])
def test_spmv_parity(request, solver, cuda, which):
    import torch

    s = request.getfixturevalue(which)
    _assemble(solver, s, cuda)
    A = O.OracleMatrix(s.n_verts, s.rows, s.cols, s.vals)
    x = np.random.default_rng(3).standard_normal(3 * s.n_verts)
    xd = to_dev(x, cuda)
    yd = torch.empty_like(xd)
    dot = solver.spmv(xd, yd, with_dot=True)
    y = yd.cpu().numpy()
    ref = A.spmv(x)
    assert np.abs(y - ref).max() <= 1e-13 * np.abs(ref).max()
    assert abs(dot - x @ ref) <= 1e-12 * abs(x @ ref)


@pytest.mark.parametrize("which", ["cube10", "cube5", "stack_small"])
def test_mixed_spmv_parity(request, solver, cuda, which):
    """The mixed PCG's SpMV (FP32 copy of the values, padded FP32 vectors, one
    vector reduction per transposed half) against the oracle's FP64 product of
    the same FP32 x: every entry within 2e-6 of (|A| |x|) -- FP32 rounding of
    the values and of at most ~30 products and sums -- and x.(A x), summed in
    FP64 from the FP32 products, within 1e-5 relative."""
    import torch

    s = request.getfixturevalue(which)
    _assemble(solver, s, cuda)
    A = O.OracleMatrix(s.n_verts, s.rows, s.cols, s.vals)
    absA = abs(A.to_scipy())
    for seed in (3, 4):
        x32 = np.random.default_rng(seed).standard_normal(3 * s.n_verts).astype(np.float32)
        x = x32.astype(np.float64)
        xd = torch.from_numpy(x32).to(cuda)
        yd = torch.full_like(xd, np.nan)
        dot = solver.spmv_mixed(xd, yd, with_dot=True)
        y = yd.double().cpu().numpy()
        ref = A.spmv(x)
        bound = 2e-6 * (absA @ np.abs(x))
        assert np.all(np.abs(y - ref) <= bound)
        assert abs(dot - x @ ref) <= 1e-5 * abs(x @ ref)
    z = torch.zeros(3 * s.n_verts, dtype=torch.float32, device=cuda)
    yz = torch.full_like(z, np.nan)
    assert solver.spmv_mixed(z, yz, with_dot=True) == 0.0
    assert not torch.any(yz != 0)


def test_stage_timing_with_and_without_graph(solver, cuda, cube10):
    """Stage timing brackets every SpMV and preconditioner apply with events,
    inside the PCG graph (external event nodes) and stream-ordered."""
    import torch

    b, A, M = _mas_setup(solver, cube10, cuda, partition_rcb(cube10.positions))
    try:
        solver.set_timing(True)
        for graph in (True, False):
            for prec in (_abi.B2S_PRECISION_FP64, _abi.B2S_PRECISION_MIXED):
                solver.reset_timers()
                x = torch.zeros_like(b)
                st = solver.pcg(b, x, tol=1e-4, stop_rule=_abi.B2S_STOP_RELRES, check_interval=5, precision=prec,
                                use_graph=graph)
                t = solver.timers()
                assert st["converged"] == 1
                assert t["spmv_launches"] >= st["iterations_exact"] > 0
                assert t["spmv_ms"] > 0 and t["precond_apply_ms"] > 0
    finally:
        solver.set_timing(False)


# ---------------------------------------------------------------------------
# MAS
# ---------------------------------------------------------------------------
def _mas_setup(solver, s, cuda, part_ids, invert_mode=_abi.B2S_INVERT_F32):
    p2r, r2p = partition_maps(part_ids)
    b = _assemble(solver, s, cuda)
    solver.mas_init(0, s.n_verts, s.adj_start, s.adj_list, p2r, r2p)
    solver.precond_assemble(_abi.B2S_PRECOND_MAS, invert_mode)
    A = O.OracleMatrix(s.n_verts, s.rows, s.cols, s.vals)
    M = O.OracleMAS(s.n_verts, s.adj_start, s.adj_list, p2r, r2p)
    M.assemble(A, 0, invert_mode)
    return b, A, M


@pytest.mark.parametrize("which", ["cube10", "stack_small"])
def test_mas_hierarchy_bit_exact(request, solver, cuda, which):
    s = request.getfixturevalue(which)
    _, A, M = _mas_setup(solver, s, cuda, partition_rcb(s.positions))
    L, total = solver.mas_info()
    assert L == M.L and total == M.total
    beg, cnt, ct = solver.mas_hierarchy(s.n_verts)
    obeg, ocnt = M.levels()
    assert np.array_equal(beg[: L + 1], obeg[: L + 1])
    assert np.array_equal(cnt[:L], ocnt[:L])
    assert np.array_equal(ct, M.coarse_table())


def test_mas_hierarchy_with_reference_metis(solver, cuda, cube10):
    if not O.metis_available():
        pytest.skip("reference METIS not compiled")
    pid = O.metis_mesh_partition(cube10.adj_start, cube10.adj_list)
    _, A, M = _mas_setup(solver, cube10, cuda, pid)
    beg, cnt, ct = solver.mas_hierarchy(cube10.n_verts)
    assert np.array_equal(ct, M.coarse_table())


@pytest.mark.parametrize("invert_mode", [_abi.B2S_INVERT_F32, _abi.B2S_INVERT_F64])
def test_mas_clusters_parity(solver, cuda, cube10, invert_mode):
    _, A, M = _mas_setup(solver, cube10, cuda, partition_rcb(cube10.positions), invert_mode)
    hess, inv = solver.mas_clusters()
    ohess, oinv = M.clusters_arrays()
    scale = np.abs(ohess).max()
    assert np.abs(hess - ohess).max() <= 1e-12 * scale
    iscale = np.abs(oinv).max()
    assert np.abs(inv.astype(np.float64) - oinv).max() <= 1e-4 * iscale


def test_mas_apply_parity(solver, cuda, cube10):
    import torch

    _, A, M = _mas_setup(solver, cube10, cuda, partition_rcb(cube10.positions))
    r = np.random.default_rng(5).standard_normal(3 * cube10.n_verts)
    rd = to_dev(r, cuda)
    zd = torch.empty_like(rd)
    solver.precond_apply(rd, zd)
    z = zd.cpu().numpy()
    ref = M.apply(r)
    assert np.abs(z - ref).max() <= 1e-4 * np.abs(ref).max()


# ---------------------------------------------------------------------------
# PCG
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("pre", [_abi.B2S_PRECOND_NONE, _abi.B2S_PRECOND_JACOBI])
@pytest.mark.parametrize("use_graph", [True, False])
def test_pcg_parity_jacobi(solver, cuda, cube10, pre, use_graph):
    import torch

    b = _assemble(solver, cube10, cuda)
    solver.precond_assemble(pre)
    A = O.OracleMatrix(cube10.n_verts, cube10.rows, cube10.cols, cube10.vals)
    x = torch.zeros_like(b)
    st = solver.pcg(b, x, tol=1e-4, stop_rule=_abi.B2S_STOP_RELRES, check_interval=1, use_graph=use_graph)
    xo, info = O.pcg(A, cube10.b, precond=pre, tol=1e-4, stop_rule=O.ORC_STOP_RELRES)
    assert st["converged"] == 1 and info["converged"] == 1
    # same algorithm, FP64 rounding differs only through the SpMV's atomics:
    # the stop fires within a couple of iterations of the oracle's
    slack = 2 if pre == _abi.B2S_PRECOND_JACOBI else max(3, info["iterations"] // 30)
    assert abs(st["iterations_exact"] - info["iterations"]) <= slack
    assert st["rel_res"] <= 1e-4 * 1.01
    xs = x.cpu().numpy()
    # two valid stops at rel-res 1e-4 (cond ~3e4) differ by up to ~1e-2 in x
    bound = 1e-3 if pre == _abi.B2S_PRECOND_JACOBI else 1e-2
    assert np.linalg.norm(xs - xo) <= bound * np.linalg.norm(xo)


def test_pcg_reference_stop_rule_and_interval(solver, cuda, cube10):
    """|r.z| <= tol |r0.z0| checked every 5 iterations, reported as the
    reference's fused solver reports it."""
    import torch

    b = _assemble(solver, cube10, cuda)
    solver.precond_assemble(_abi.B2S_PRECOND_JACOBI)
    A = O.OracleMatrix(cube10.n_verts, cube10.rows, cube10.cols, cube10.vals)
    x = torch.zeros_like(b)
    st = solver.pcg(b, x, tol=1e-3, stop_rule=_abi.B2S_STOP_RZ, check_interval=5)
    _, info = O.pcg(A, cube10.b, precond=O.ORC_PRECOND_JACOBI, tol=1e-3, stop_rule=O.ORC_STOP_RZ, check_interval=5)
    assert st["iterations"] == info["iterations"] and st["iterations"] % 5 == 0
    assert abs(st["rz0"] - info["rz0"]) <= 1e-12 * abs(info["rz0"])


@pytest.mark.parametrize("which", ["cube10", "stack_small"])
def test_pcg_mas_parity(request, solver, cuda, which):
    import torch

    s = request.getfixturevalue(which)
    b, A, M = _mas_setup(solver, s, cuda, partition_rcb(s.positions))
    x = torch.zeros_like(b)
    st = solver.pcg(b, x, tol=1e-4, stop_rule=_abi.B2S_STOP_RELRES, check_interval=1)
    xo, info = O.pcg(A, s.b, precond=O.ORC_PRECOND_MAS, mas=M, tol=1e-4, stop_rule=O.ORC_STOP_RELRES)
    assert st["converged"] == 1 and info["converged"] == 1
    assert abs(st["iterations_exact"] - info["iterations"]) <= 2
    assert st["rel_res"] <= 1e-4 * 1.01


@pytest.mark.parametrize("pre", [_abi.B2S_PRECOND_JACOBI, _abi.B2S_PRECOND_MAS])
def test_solution_parity_tight_tolerance(solver, cuda, cube10, pre):
    """At a matched tight tolerance the GPU solution agrees with the FP64
    direct solution within 1e-6 relative."""
    import scipy.sparse.linalg as spla
    import torch

    if pre == _abi.B2S_PRECOND_MAS:
        b, A, M = _mas_setup(solver, cube10, cuda, partition_rcb(cube10.positions))
    else:
        b = _assemble(solver, cube10, cuda)
        solver.precond_assemble(pre)
        A = O.OracleMatrix(cube10.n_verts, cube10.rows, cube10.cols, cube10.vals)
    x = torch.zeros_like(b)
    st = solver.pcg(b, x, tol=1e-11, stop_rule=_abi.B2S_STOP_RELRES, check_interval=5)
    xt = spla.spsolve(A.to_scipy().tocsc(), cube10.b)
    assert st["converged"] == 1
    assert np.linalg.norm(x.cpu().numpy() - xt) <= 1e-6 * np.linalg.norm(xt)


def test_pcg_warm_start(solver, cuda, cube10):
    import torch

    b = _assemble(solver, cube10, cuda)
    solver.precond_assemble(_abi.B2S_PRECOND_JACOBI)
    x = torch.zeros_like(b)
    st0 = solver.pcg(b, x, tol=1e-8, stop_rule=_abi.B2S_STOP_RELRES, check_interval=1)
    x2 = x.clone()
    st1 = solver.pcg(b, x2, tol=1e-8, stop_rule=_abi.B2S_STOP_RELRES, check_interval=1, x0_given=True)
    assert st1["iterations_exact"] <= 1
    assert st1["rel_res"] <= 1e-8 * 1.01


def test_pcg_zero_rhs(solver, cuda, cube5):
    import torch

    b = _assemble(solver, cube5, cuda)
    solver.precond_assemble(_abi.B2S_PRECOND_JACOBI)
    z = torch.zeros_like(b)
    x = torch.ones_like(b)
    st = solver.pcg(z, x, tol=1e-4)
    assert st["converged"] == 1 and st["iterations"] == 0
    assert float(x.abs().max()) == 0.0


def test_calls_out_of_order_are_state_errors(solver, cuda):
    import torch

    from libuipc_b200.linear_system import B200SolveError

    v = torch.zeros(9, dtype=torch.float64, device=cuda)
    with pytest.raises(B200SolveError) as ei:
        solver.pcg(v, v.clone())
    assert ei.value.code == _abi.B2S_ERR_STATE
    with pytest.raises(B200SolveError):
        solver.precond_apply(v, v.clone())


# ---------------------------------------------------------------------------
# mixed precision
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("which", ["cube10", "stack_small"])
@pytest.mark.parametrize("pre", [_abi.B2S_PRECOND_JACOBI, _abi.B2S_PRECOND_MAS])
def test_mixed_pcg_fp64_verified(request, solver, cuda, which, pre):
    """FP32 matrix/vectors + BF16 MAS inverses + FP64 dots: the stop is
    confirmed by the FP64 residual, and the iteration count stays close to the
    plain FP64 solve's."""
    import torch

    s = request.getfixturevalue(which)
    if pre == _abi.B2S_PRECOND_MAS:
        b, A, M = _mas_setup(solver, s, cuda, partition_rcb(s.positions))
    else:
        b = _assemble(solver, s, cuda)
        solver.precond_assemble(pre)
    x64 = torch.zeros_like(b)
    plain = solver.pcg(b, x64, tol=1e-4, stop_rule=_abi.B2S_STOP_RELRES, check_interval=5)
    x = torch.zeros_like(b)
    st = solver.pcg(b, x, tol=1e-4, stop_rule=_abi.B2S_STOP_RELRES, check_interval=5,
                    precision=_abi.B2S_PRECISION_MIXED, replace_every=50)
    assert st["converged"] == 1
    assert st["rel_res"] <= 1e-4
    assert st["iterations_exact"] <= 1.25 * plain["iterations_exact"] + 5
    assert np.linalg.norm(x.cpu().numpy() - x64.cpu().numpy()) <= 2e-2 * np.linalg.norm(x64.cpu().numpy())


def test_mixed_pcg_tight_tolerance_by_residual_replacement(solver, cuda, cube10):
    """FP64 residual replacement wins back accuracy beyond FP32: the mixed
    solve reaches rel-res 1e-9 and the FP64 direct solution within 1e-6."""
    import scipy.sparse.linalg as spla
    import torch

    b, A, M = _mas_setup(solver, cube10, cuda, partition_rcb(cube10.positions))
    x = torch.zeros_like(b)
    st = solver.pcg(b, x, tol=1e-9, stop_rule=_abi.B2S_STOP_RELRES, check_interval=5,
                    precision=_abi.B2S_PRECISION_MIXED, replace_every=20)
    assert st["converged"] == 1 and st["rel_res"] <= 1e-9
    assert st["replacements"] >= 1
    xt = spla.spsolve(A.to_scipy().tocsc(), cube10.b)
    assert np.linalg.norm(x.cpu().numpy() - xt) <= 1e-6 * np.linalg.norm(xt)


@pytest.mark.parametrize("which", ["cube10", "stack_small"])
def test_mixed_mas_apply_matches_oracle_bf16(request, solver, cuda, which):
    """Tensor-core apply of the BF16 diagonal-scaled inverses against the
    oracle's apply with the same BF16 entries (the oracle is given the
    device's FP32 inverses and quantises them as the device does): they differ only by the FP32
    accumulation order and the ~16-bit (hi + lo BF16) residual operand, so
    relative 1e-4 in norm and 1e-3 of max|z| per entry."""
    import torch

    s = request.getfixturevalue(which)
    b, A, M = _mas_setup(solver, s, cuda, partition_rcb(s.positions))
    # the oracle quantises the device's FP32 inverses (same BF16 entries)
    M.set_inverses(solver.mas_clusters()[1])
    M.quantize(2)
    rng = np.random.default_rng(21)
    for trial in range(3):
        r = rng.standard_normal(3 * s.n_verts) * (10.0 ** (3 * trial))
        zr = M.apply(r)
        r32 = torch.tensor(r, dtype=torch.float32, device=cuda)
        z32 = torch.zeros_like(r32)
        solver.precond_apply_mixed(r32, z32)
        z = z32.double().cpu().numpy()
        assert np.linalg.norm(z - zr) <= 1e-4 * np.linalg.norm(zr)
        assert np.max(np.abs(z - zr)) <= 1e-3 * np.max(np.abs(zr))


def test_mixed_spmv_bf16_apply_consistent(solver, cuda, cube10):
    """The mixed path's BF16 MAS apply stays within BF16 rounding of the FP32
    apply (relative 2e-2 in the worst entry, 5e-3 in norm)."""
    import torch

    b, A, M = _mas_setup(solver, cube10, cuda, partition_rcb(cube10.positions))
    # run one mixed solve so the BF16 inverses are packed, then compare the
    # FP32 apply of the oracle to the oracle with BF16-quantised inverses
    M2 = O.OracleMAS(cube10.n_verts, cube10.adj_start, cube10.adj_list, *partition_maps(partition_rcb(cube10.positions)))
    M2.assemble(A, 0, 0)
    M2.quantize(2)
    r = np.random.default_rng(9).standard_normal(3 * cube10.n_verts)
    z32 = M.apply(r)
    z16 = M2.apply(r)
    assert np.linalg.norm(z16 - z32) <= 5e-3 * np.linalg.norm(z32)
    x = torch.zeros_like(b)
    st = solver.pcg(b, x, tol=1e-4, stop_rule=_abi.B2S_STOP_RELRES, precision=_abi.B2S_PRECISION_MIXED)
    assert st["converged"] == 1


def test_spmv_timing_utility(solver, cuda, cube10):
    """b2s_spmv_mixed_timing: a positive average launch time, and the solver
    still solves the assembled system afterwards (the batch writes only its
    own scratch)."""
    import torch

    from libuipc_b200 import _abi
    from libuipc_b200.linear_system import partition_maps, partition_rcb

    s = cube10
    solver.assemble(s.n_verts, to_dev(s.rows, cuda), to_dev(s.cols, cuda), to_dev(s.vals, cuda))
    ms = solver.spmv_mixed_timing(20)
    assert 0.0 < ms < 10.0
    p2r, r2p = partition_maps(partition_rcb(s.positions))
    solver.mas_init(0, s.n_verts, s.adj_start, s.adj_list, p2r, r2p)
    solver.precond_assemble(_abi.B2S_PRECOND_MAS)
    b = to_dev(s.b, cuda)
    x = torch.zeros_like(b)
    st = solver.pcg(b, x, tol=1e-6, stop_rule=_abi.B2S_STOP_RELRES, precision=_abi.B2S_PRECISION_MIXED,
                    replace_every=20)
    assert st["converged"] == 1


def test_mas_on_the_graph_partition(solver, cuda, cube10):
    """The MAS built on b2s_partition_graph's parts (connectivity only, the
    drop-in for mesh_partition's METIS call): the hierarchy equals the
    oracle's on the same partition and the FP64 MAS-PCG stops within 2
    iterations of the oracle's."""
    import torch

    from libuipc_b200 import _abi
    from libuipc_b200.linear_system import partition_graph, partition_maps
    from oracle import oracle as O

    s = cube10
    p2r, r2p = partition_maps(partition_graph(s.adj_start, s.adj_list))
    solver.assemble(s.n_verts, to_dev(s.rows, cuda), to_dev(s.cols, cuda), to_dev(s.vals, cuda))
    solver.mas_init(0, s.n_verts, s.adj_start, s.adj_list, p2r, r2p)
    solver.precond_assemble(_abi.B2S_PRECOND_MAS)
    A = O.OracleMatrix(s.n_verts, s.rows, s.cols, s.vals)
    M = O.OracleMAS(s.n_verts, s.adj_start, s.adj_list, p2r, r2p)
    M.assemble(A, 0, 0)
    beg, cnt, ct = solver.mas_hierarchy(s.n_verts)
    obeg, ocnt = M.levels()
    L, _ = solver.mas_info()
    assert np.array_equal(beg[: L + 1], obeg[: L + 1]) and np.array_equal(ct, M.coarse_table())
    _, info = O.pcg(A, s.b, precond=O.ORC_PRECOND_MAS, mas=M, tol=1e-6, stop_rule=O.ORC_STOP_RELRES)
    b = to_dev(s.b, cuda)
    x = torch.zeros_like(b)
    st = solver.pcg(b, x, tol=1e-6, stop_rule=_abi.B2S_STOP_RELRES, check_interval=1)
    assert st["converged"] == 1 and info["converged"] == 1
    assert abs(st["iterations_exact"] - info["iterations"]) <= 2
