"""The caller side of the solve as libuipc's GlobalLinearSystem runs it: linear
subsystems report their extents, the DoF and triplet ranges are laid out, the
triplet arrays are filled, and every subsystem writes into its own sub-range.

Follows src/backends/cuda/linear_system/global_linear_system.cu:
  * init (:120-175): diagonal subsystems sorted by uid, off-diagonal ones by uid;
    the diagonal ones take the first triplet ranges, the couplings follow;
  * _update_subsystem_extent (:321-405): per diagonal subsystem a DoF count and a
    Hessian block count, per coupling the lr and rl block counts (its range holds
    lr then rl); exclusive scans give the offsets; storage grows to 1.1x the
    total when the total exceeds the capacity (reserve_ratio,
    global_linear_system.h:287) and never shrinks;
  * _assemble_linear_system (:407-497): row and column indices filled with -1
    (the assembly drops rows < 0, so an unwritten slot disappears), b with 0;
    a diagonal subsystem writes its gradient into b[dof_offset, +dof_count) and
    its block triplets into its range with the block offset (dof_offset/3,
    dof_offset/3); a coupling writes lr blocks at (l_offset, r_offset) and rl
    blocks at (r_offset, l_offset) (TripletMatrixView::subview / submatrix,
    cuda_tool/linear_system/views.h:77-88);
  * distribute_solution (:531-544): each diagonal subsystem receives the
    solution x of A x = b on its DoF range (SolutionInfo::solution) and turns
    it into its own displacement, dx = -x (FEMLinearSubsystem's
    retrieve_solution kernel, finite_element/fem_linear_subsystem.cu:119-126).

The arrays are torch tensors (any device) or numpy arrays; a subsystem writes
with ``write`` (one block) or ``write_many`` (vectorised).
"""
from __future__ import annotations

DOF_BLOCK = 3
RESERVE_RATIO = 1.1


class DiagExtentInfo:
    """GlobalLinearSystem::DiagExtentInfo: ``extent(hessian_block_count, dof_count)``."""

    def __init__(self):
        self.block_count = 0
        self.dof_count = 0

    def extent(self, hessian_block_count: int, dof_count: int):
        if dof_count % DOF_BLOCK:
            raise ValueError("a subsystem's DoF count must be a multiple of 3")
        self.block_count, self.dof_count = int(hessian_block_count), int(dof_count)


class OffDiagExtentInfo:
    """GlobalLinearSystem::OffDiagExtentInfo: ``extent(lr_block_count, rl_block_count)``."""

    def __init__(self):
        self.lr_block_count = 0
        self.rl_block_count = 0

    def extent(self, lr_block_count: int, rl_block_count: int):
        self.lr_block_count, self.rl_block_count = int(lr_block_count), int(rl_block_count)


class TripletView:
    """A triplet sub-range [offset, offset + count) of the global arrays seen as a
    block matrix of ``shape`` blocks placed at block ``origin``: a write of block
    (i, j) into slot k stores (origin[0] + i, origin[1] + j, H) at offset + k."""

    def __init__(self, rows, cols, vals, offset: int, count: int, origin, shape):
        self.rows, self.cols, self.vals = rows, cols, vals
        self.offset, self.count = int(offset), int(count)
        self.origin = (int(origin[0]), int(origin[1]))
        self.shape = (int(shape[0]), int(shape[1]))

    def write(self, k: int, i: int, j: int, H):
        """Block (i, j) into slot k; H: 9 values, column-major (Eigen::Matrix3d)."""
        if not (0 <= k < self.count):
            raise IndexError(f"triplet slot {k} outside [0, {self.count})")
        if not (0 <= i < self.shape[0] and 0 <= j < self.shape[1]):
            raise IndexError(f"block ({i}, {j}) outside the {self.shape[0]} x {self.shape[1]} submatrix")
        s = self.offset + k
        self.rows[s] = self.origin[0] + i
        self.cols[s] = self.origin[1] + j
        self.vals[s] = _as_like(self.vals, H).reshape(9)

    def write_many(self, k0: int, i, j, H):
        """Blocks (i[t], j[t]) into slots k0 + t; H: [m, 9] column-major."""
        m = len(i)
        if m == 0:
            return
        if k0 < 0 or k0 + m > self.count:
            raise IndexError(f"triplet slots [{k0}, {k0 + m}) outside [0, {self.count})")
        ii, jj = _as_like(self.rows, i), _as_like(self.cols, j)
        if int(ii.min()) < 0 or int(ii.max()) >= self.shape[0] or int(jj.min()) < 0 or int(jj.max()) >= self.shape[1]:
            raise IndexError(f"blocks outside the {self.shape[0]} x {self.shape[1]} submatrix")
        s = slice(self.offset + k0, self.offset + k0 + m)
        self.rows[s] = ii + self.origin[0]
        self.cols[s] = jj + self.origin[1]
        self.vals[s] = _as_like(self.vals, H).reshape(m, 9)


class DenseView:
    """A sub-range [offset, offset + count) of a vector."""

    def __init__(self, v, offset: int, count: int):
        self.v, self.offset, self.count = v, int(offset), int(count)

    def view(self):
        return self.v[self.offset:self.offset + self.count]


class DiagInfo:
    """GlobalLinearSystem::DiagInfo: ``hessians()`` and ``gradients()`` of one
    diagonal subsystem."""

    def __init__(self, hessians: TripletView, gradients: DenseView):
        self._h, self._g = hessians, gradients

    def hessians(self) -> TripletView:
        return self._h

    def gradients(self):
        """The subsystem's slice of b (a view: writes land in b)."""
        return self._g.view()

    def write_gradients(self, g):
        """b on the subsystem's DoF range = g (any array type)."""
        v = self._g.view()
        v[:] = _as_like(v, g).reshape(v.shape)


class OffDiagInfo:
    """GlobalLinearSystem::OffDiagInfo: ``lr_hessian()`` and ``rl_hessian()``."""

    def __init__(self, lr: TripletView, rl: TripletView):
        self._lr, self._rl = lr, rl

    def lr_hessian(self) -> TripletView:
        return self._lr

    def rl_hessian(self) -> TripletView:
        return self._rl


class SolutionInfo:
    """GlobalLinearSystem::SolutionInfo: ``solution()`` = x, the solution of
    A x = b, on the subsystem's DoF range; the subsystem negates it into its
    displacement dx = -x, as the reference's subsystems do."""

    def __init__(self, x):
        self._x = x

    def solution(self):
        return self._x


class DiagLinearSubsystem:
    """A diagonal subsystem (DiagLinearSubsystem, diag_linear_subsystem.h:33-76):
    override ``report_extent``, ``assemble`` and (optionally) ``retrieve_solution``."""

    def __init__(self, uid: int):
        self.uid = int(uid)
        self.dof_offset = 0
        self.dof_count = 0

    def report_extent(self, info: DiagExtentInfo):
        raise NotImplementedError

    def assemble(self, info: DiagInfo):
        raise NotImplementedError

    def retrieve_solution(self, info: SolutionInfo):
        pass


class OffDiagLinearSubsystem:
    """A coupling between two diagonal subsystems (OffDiagLinearSubsystem):
    ``l`` and ``r`` are the diagonal subsystems of its block rows and columns."""

    def __init__(self, uid: int, l: DiagLinearSubsystem, r: DiagLinearSubsystem):
        self.uid, self.l, self.r = int(uid), l, r

    def report_extent(self, info: OffDiagExtentInfo):
        raise NotImplementedError

    def assemble(self, info: OffDiagInfo):
        raise NotImplementedError


class SubsystemLayout:
    """The DoF and triplet ranges of a set of subsystems, recomputed every
    Newton iteration by ``update``."""

    def __init__(self, diag, off_diag=()):
        self.diag = sorted(diag, key=lambda d: d.uid)
        self.off_diag = sorted(off_diag, key=lambda o: o.uid)
        for o in self.off_diag:
            if o.l not in self.diag or o.r not in self.diag:
                raise ValueError("a coupling's subsystems must be among the diagonal subsystems")
        self.dof_offsets, self.dof_counts = [], []
        self.triplet_offsets, self.triplet_counts = [], []
        self.lr_counts = []
        self.total_dof = self.total_triplets = 0
        self.dof_capacity = self.triplet_capacity = 0

    def update(self):
        """Report every extent, scan the offsets, grow the capacities; returns
        (total DoF, total triplets)."""
        counts = []
        self.dof_counts = []
        for d in self.diag:
            e = DiagExtentInfo()
            d.report_extent(e)
            self.dof_counts.append(e.dof_count)
            counts.append(e.block_count)
        self.lr_counts = []
        for o in self.off_diag:
            e = OffDiagExtentInfo()
            o.report_extent(e)
            self.lr_counts.append((e.lr_block_count, e.rl_block_count))
            counts.append(e.lr_block_count + e.rl_block_count)
        self.dof_offsets = _exclusive_scan(self.dof_counts)
        self.triplet_counts = counts
        self.triplet_offsets = _exclusive_scan(counts)
        self.total_dof = sum(self.dof_counts)
        self.total_triplets = sum(counts)
        for d, off, cnt in zip(self.diag, self.dof_offsets, self.dof_counts):
            d.dof_offset, d.dof_count = off, cnt
        if self.total_dof > self.dof_capacity:
            self.dof_capacity = int(self.total_dof * RESERVE_RATIO)
        if self.total_triplets > self.triplet_capacity:
            self.triplet_capacity = int(self.total_triplets * RESERVE_RATIO)
        return self.total_dof, self.total_triplets

    @property
    def n_block_rows(self) -> int:
        return self.total_dof // DOF_BLOCK

    def assemble(self, rows, cols, vals, b):
        """Fill rows / cols with -1 and b with 0 over the current totals, then let
        every subsystem write its range (diagonal subsystems first)."""
        T, n = self.total_triplets, self.total_dof
        rows[:T] = -1
        cols[:T] = -1
        b[:n] = 0
        for idx, d in enumerate(self.diag):
            blk = self.dof_offsets[idx] // DOF_BLOCK
            nblk = self.dof_counts[idx] // DOF_BLOCK
            h = TripletView(rows, cols, vals, self.triplet_offsets[idx], self.triplet_counts[idx], (blk, blk),
                            (nblk, nblk))
            d.assemble(DiagInfo(h, DenseView(b, self.dof_offsets[idx], self.dof_counts[idx])))
        nd = len(self.diag)
        for k, o in enumerate(self.off_diag):
            li, ri = self.diag.index(o.l), self.diag.index(o.r)
            lb, ln = self.dof_offsets[li] // DOF_BLOCK, self.dof_counts[li] // DOF_BLOCK
            rb, rn = self.dof_offsets[ri] // DOF_BLOCK, self.dof_counts[ri] // DOF_BLOCK
            lr, rl = self.lr_counts[k]
            off = self.triplet_offsets[nd + k]
            o.assemble(OffDiagInfo(TripletView(rows, cols, vals, off, lr, (lb, rb), (ln, rn)),
                                   TripletView(rows, cols, vals, off + lr, rl, (rb, lb), (rn, ln))))

    def distribute(self, x):
        """Each diagonal subsystem receives the solution x on its DoF range
        (it negates it into dx itself)."""
        for d, off, cnt in zip(self.diag, self.dof_offsets, self.dof_counts):
            d.retrieve_solution(SolutionInfo(x[off:off + cnt]))


def _exclusive_scan(counts):
    out, acc = [], 0
    for c in counts:
        out.append(acc)
        acc += c
    return out


def _as_like(dst, v):
    """``v`` as the array type of ``dst`` (torch tensor on dst's device or numpy)."""
    try:
        import torch

        if isinstance(dst, torch.Tensor):
            return torch.as_tensor(v, dtype=dst.dtype, device=dst.device)
    except ImportError:
        pass
    import numpy as np

    return np.asarray(v, dtype=dst.dtype)
