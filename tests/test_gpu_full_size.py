"""Size-independent properties at the headline workload's full size -- 8
stacked 40^3-cell tet cubes, 551,368 block rows, 31.5 M raw triplets, first
Newton system from rest -- where the oracle cannot follow in seconds:

* assembly: row pointers monotone, every row starting at its diagonal block,
  columns strictly increasing and upper, and a checksum: the stored blocks sum
  to the kept (row >= 0, row <= col) triplets (FP64, 1e-12 of the absolute sum);
* SpMV: x.(A y) = y.(A x) (1e-12 of |x| |A y|), the fused dot equals x.(A x),
  and the mixed SpMV (FP32 values and vectors) within 1e-4 of the FP64 one in
  norm (FP32 rounding of ~30 products per entry, ~2e-6 of |A||x|, with room for
  the cancellation a stiff row has at this size);
* MAS (RCB partition): r1.(P r2) = r2.(P r1) and P linear (FP32 apply: 1e-5),
  r.(P r) > 0;
* mixed PCG: converged, and the residual b - A x recomputed here by the FP64
  SpMV is below 1e-4 of |b|."""
import numpy as np
import pytest

from libuipc_b200 import _abi
from libuipc_b200.linear_system import partition_maps, partition_rcb

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def full_stack():
    from libuipc_b200 import scene

    return scene.generate(scene=1, cells_x=40, cells_y=40, cells_z=40, n_cubes=8, seed=0)


def test_full_size_properties(solver, cuda, full_stack):
    import torch

    s = full_stack
    assert s.n_verts == 551_368
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)  # noqa: E731
    solver.assemble(s.n_verts, dev(s.rows), dev(s.cols), dev(s.vals))
    nb, U = solver.matrix_info()
    rp, col, val = solver.upper_bsr()
    assert nb == s.n_verts and rp[0] == 0 and rp[-1] == U
    assert np.all(np.diff(rp) >= 1)
    assert np.array_equal(col[rp[:-1]], np.arange(nb))  # the diagonal block leads every row
    row_of = np.repeat(np.arange(nb, dtype=np.int64), np.diff(rp))
    same = row_of[1:] == row_of[:-1]
    assert np.all(np.diff(col.astype(np.int64))[same] > 0)
    assert np.all(col >= row_of) and np.all(col < nb)
    keep = (s.rows >= 0) & (s.rows <= s.cols)
    kept = s.vals[keep]
    scale = np.abs(kept).sum(axis=0)
    assert np.all(np.abs(val.sum(axis=0) - kept.sum(axis=0)) <= 1e-12 * scale)
    del kept, val

    g = torch.Generator().manual_seed(5)
    n = 3 * nb
    x = torch.randn(n, dtype=torch.float64, generator=g).to(cuda)
    y = torch.randn(n, dtype=torch.float64, generator=g).to(cuda)
    Ax, Ay = torch.empty_like(x), torch.empty_like(x)
    dot = solver.spmv(x, Ax, with_dot=True)
    solver.spmv(y, Ay)
    lhs, rhs = float(x @ Ay), float(y @ Ax)
    assert abs(lhs - rhs) <= 1e-12 * float(x.norm() * Ay.norm())
    xAx = float(x @ Ax)
    assert abs(dot - xAx) <= 1e-12 * abs(xAx)
    x32 = x.float()
    y32 = torch.full_like(x32, float("nan"))
    solver.spmv_mixed(x32, y32)
    ref = torch.empty_like(x)
    solver.spmv(x32.double(), ref)
    assert float((y32.double() - ref).norm()) <= 1e-4 * float(ref.norm())

    p2r, r2p = partition_maps(partition_rcb(s.positions))
    solver.mas_init(0, nb, s.adj_start, s.adj_list, p2r, r2p)
    solver.precond_assemble(_abi.B2S_PRECOND_MAS, _abi.B2S_INVERT_SWEEP_F32)
    P = lambda r: (lambda z: (solver.precond_apply(r, z), z)[1])(torch.empty_like(r))  # noqa: E731
    z1, z2 = P(x), P(y)
    a, c = float(y @ z1), float(x @ z2)
    assert abs(a - c) <= 1e-5 * float(x.norm() * z2.norm())
    assert float(x @ z1) > 0 and float(y @ z2) > 0
    z3 = P(2.0 * x + y)
    assert float((z3 - (2.0 * z1 + z2)).norm()) <= 1e-5 * float(z3.norm())

    b = torch.from_numpy(s.b).to(cuda)
    sol = torch.zeros_like(b)
    st = solver.pcg(b, sol, tol=1e-4, stop_rule=_abi.B2S_STOP_RELRES, check_interval=5,
                    precision=_abi.B2S_PRECISION_MIXED, replace_every=50)
    assert st["converged"] == 1
    As = torch.empty_like(b)
    solver.spmv(sol, As)
    assert float((b - As).norm()) <= 1e-4 * float(b.norm())
