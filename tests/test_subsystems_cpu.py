"""The caller side of the solve (libuipc_b200/subsystems.py) on CPU: subsystem
order by uid (diagonal first), DoF and triplet offsets by exclusive scans,
capacity grown by 1.1 and never shrunk, the -1 / 0 fill, block offsets of the
diagonal and coupling sub-ranges, and the assembled matrix (through the oracle,
which drops the unwritten slots like the reference's converter) equal to the
dense matrix the subsystems describe."""
import numpy as np
import pytest

from libuipc_b200.subsystems import DiagLinearSubsystem, OffDiagLinearSubsystem, SubsystemLayout
from oracle import oracle as O


def _spd(n, rng, scale=1.0):
    a = rng.standard_normal((n, n))
    return scale * (a @ a.T + n * np.eye(n))


class Body(DiagLinearSubsystem):
    """12 DoF (4 block rows), the full 12x12 block written as 16 upper-first
    triplets with the lower 3x3 blocks zeroed (abd_linear_subsystem.cu:21-31)."""

    def __init__(self, uid, H, g, spare=0):
        super().__init__(uid)
        self.H, self.g, self.spare = H, g, spare
        self.dx = None

    def report_extent(self, info):
        info.extent(16 + self.spare, 12)

    def assemble(self, info):
        h = info.hessians()
        k = 0
        for bi in range(4):
            for bj in range(4):
                B = self.H[3 * bi:3 * bi + 3, 3 * bj:3 * bj + 3] if bi <= bj else np.zeros((3, 3))
                h.write(k, bi, bj, B.T.reshape(9))  # column-major
                k += 1
        info.write_gradients(self.g)

    def retrieve_solution(self, info):
        # as FEMLinearSubsystem / ABDLinearSubsystem: dx = -x
        self.dx = -info.solution()


class Mesh(DiagLinearSubsystem):
    """nv vertices, block-upper triplets given as arrays (local ids)."""

    def __init__(self, uid, nv, r, c, vals, g):
        super().__init__(uid)
        self.nv, self.r, self.c, self.vals, self.g = nv, r, c, vals, g
        self.dx = None

    def report_extent(self, info):
        info.extent(len(self.r), 3 * self.nv)

    def assemble(self, info):
        info.hessians().write_many(0, self.r, self.c, self.vals)
        info.write_gradients(self.g)

    def retrieve_solution(self, info):
        # as FEMLinearSubsystem / ABDLinearSubsystem: dx = -x
        self.dx = -info.solution()


class Coupling(OffDiagLinearSubsystem):
    """lr blocks (body row, mesh column) written; rl range reserved and left
    unwritten (the assembly keeps the upper part only)."""

    def __init__(self, uid, l, r, blocks, n_rl=0):
        super().__init__(uid, l, r)
        self.blocks, self.n_rl = blocks, n_rl

    def report_extent(self, info):
        info.extent(len(self.blocks), self.n_rl)

    def assemble(self, info):
        lr = info.lr_hessian()
        for k, (i, j, B) in enumerate(self.blocks):
            lr.write(k, i, j, B.T.reshape(9))


def _scene(rng):
    body = Body(0, _spd(12, rng), rng.standard_normal(12), spare=2)
    nv = 5
    A = _spd(3 * nv, rng)
    r, c, v = [], [], []
    for i in range(nv):
        for j in range(i, nv):
            if j - i <= 1:
                r.append(i)
                c.append(j)
                v.append(A[3 * i:3 * i + 3, 3 * j:3 * j + 3].T.reshape(9))
    mesh = Mesh(1, nv, np.array(r), np.array(c), np.array(v), rng.standard_normal(3 * nv))
    blocks = [(1, 2, 0.01 * rng.standard_normal((3, 3))), (3, 4, 0.01 * rng.standard_normal((3, 3)))]
    coup = Coupling(5, body, mesh, blocks, n_rl=1)
    return body, mesh, coup, A


def _expected_dense(body, mesh, coup, A):
    n = 12 + 3 * mesh.nv
    D = np.zeros((n, n))
    D[:12, :12] = body.H
    for i, j, v in zip(mesh.r, mesh.c, mesh.vals):
        B = v.reshape(3, 3).T
        D[12 + 3 * i:15 + 3 * i, 12 + 3 * j:15 + 3 * j] = B
        if i != j:
            D[12 + 3 * j:15 + 3 * j, 12 + 3 * i:15 + 3 * i] = B.T
    for i, j, B in coup.blocks:
        D[3 * i:3 * i + 3, 12 + 3 * j:15 + 3 * j] = B
        D[12 + 3 * j:15 + 3 * j, 3 * i:3 * i + 3] = B.T
    return D


def test_layout_order_offsets_and_capacity():
    rng = np.random.default_rng(1)
    body, mesh, coup, _ = _scene(rng)
    lay = SubsystemLayout([mesh, body], [coup])  # given out of uid order
    assert [d.uid for d in lay.diag] == [0, 1]
    n, T = lay.update()
    assert n == 12 + 15 and lay.n_block_rows == 9
    assert lay.dof_offsets == [0, 12] and (body.dof_offset, mesh.dof_offset) == (0, 12)
    nm = len(mesh.r)
    assert lay.triplet_counts == [18, nm, 3] and lay.triplet_offsets == [0, 18, 18 + nm]
    assert T == 21 + nm and lay.triplet_capacity == int(T * 1.1) and lay.dof_capacity == int(n * 1.1)
    cap = lay.triplet_capacity
    body.spare = 0  # fewer triplets: the capacity stays
    assert lay.update()[1] == T - 2 and lay.triplet_capacity == cap
    body.spare = 40  # more than the capacity: grows to 1.1x
    T2 = lay.update()[1]
    assert lay.triplet_capacity == int(T2 * 1.1) > cap


def test_fill_offsets_and_assembled_matrix():
    rng = np.random.default_rng(2)
    body, mesh, coup, A = _scene(rng)
    lay = SubsystemLayout([body, mesh], [coup])
    n, T = lay.update()
    rows = np.full(lay.triplet_capacity, 77, np.int32)
    cols = np.full(lay.triplet_capacity, 77, np.int32)
    vals = np.zeros((lay.triplet_capacity, 9))
    b = np.full(lay.dof_capacity, 5.0)
    lay.assemble(rows, cols, vals, b)
    # unwritten slots: the body's 2 spare ones and the coupling's rl one
    assert list(rows[16:18]) == [-1, -1] and list(cols[16:18]) == [-1, -1]
    assert rows[T - 1] == -1 and cols[T - 1] == -1
    # block offsets: mesh rows start at block 4, coupling rows are body rows, columns mesh columns
    nm = len(mesh.r)
    assert np.array_equal(rows[18:18 + nm], mesh.r + 4) and np.array_equal(cols[18:18 + nm], mesh.c + 4)
    assert list(rows[18 + nm:20 + nm]) == [1, 3] and list(cols[18 + nm:20 + nm]) == [2 + 4, 4 + 4]
    assert np.array_equal(b[:12], body.g) and np.array_equal(b[12:n], mesh.g)
    M = O.OracleMatrix(lay.n_block_rows, rows[:T], cols[:T], vals[:T]).to_scipy().toarray()
    assert np.array_equal(M, _expected_dense(body, mesh, coup, A))


def test_writes_are_range_checked_and_solution_is_distributed():
    import torch

    rng = np.random.default_rng(3)
    body, mesh, coup, _ = _scene(rng)
    lay = SubsystemLayout([body, mesh], [coup])
    n, T = lay.update()
    rows = torch.zeros(lay.triplet_capacity, dtype=torch.int32)
    cols = torch.zeros_like(rows)
    vals = torch.zeros((lay.triplet_capacity, 9), dtype=torch.float64)
    b = torch.zeros(lay.dof_capacity, dtype=torch.float64)
    lay.assemble(rows, cols, vals, b)  # torch tensors work the same
    assert int(rows[16]) == -1 and int(rows[18]) == int(mesh.r[0]) + 4
    from libuipc_b200.subsystems import TripletView

    v = TripletView(rows, cols, vals, 18, 3, (4, 4), (5, 5))
    with pytest.raises(IndexError):
        v.write(0, 5, 0, np.zeros(9))  # block row outside the submatrix
    with pytest.raises(IndexError):
        v.write(3, 0, 0, np.zeros(9))  # slot outside the range
    with pytest.raises(IndexError):
        v.write_many(1, [0, 1, 2], [0, 0, 0], np.zeros((3, 9)))
    x = np.arange(n, dtype=np.float64)
    lay.distribute(x)  # the solution of A x = b; each subsystem negates it
    assert np.array_equal(body.dx, -x[:12]) and np.array_equal(mesh.dx, -x[12:])
