"""The PCG's failure arms, driven by host-made inputs (no GPU fault involved).

* PSD guard (LinearFusedPCG::fused_pcg, linear_fused_pcg.cu:1843-1877): when
  r0.z0 < 0 or is not finite the preconditioner is bypassed and plain CG runs.
  A negated SPD system (A' = -A, b' = -b: the same solution) makes every
  block-Jacobi action negative definite, so r0.z0 < 0.
* Non-finite input (linear_fused_pcg.cu:1013-1060): a NaN in b is refused
  with B2S_ERR_NUMERIC before any iteration.
* Iteration cap (LinearPCG::pcg, linear_pcg.cu:420-435): with max_iter = 3 the
  solve stops unconverged and reports it.
* Warm start refused by its FP64 check: x0 = 0 (the plain start).
"""
import numpy as np
import pytest

from conftest import to_dev
from libuipc_b200 import _abi
from libuipc_b200.linear_system import B200SolveError, partition_maps, partition_rcb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PRECISIONS = [_abi.B2S_PRECISION_FP64, _abi.B2S_PRECISION_MIXED]


def _setup(solver, s, dev, kind, negate=False):
    sign = -1.0 if negate else 1.0
    solver.assemble(s.n_verts, to_dev(s.rows, dev), to_dev(s.cols, dev), to_dev(sign * s.vals, dev))
    if kind == _abi.B2S_PRECOND_MAS:
        p2r, r2p = partition_maps(partition_rcb(s.positions))
        solver.mas_init(0, s.n_verts, s.adj_start, s.adj_list, p2r, r2p)
    solver.precond_assemble(kind)
    return to_dev(sign * s.b, dev)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_psd_guard_bypasses_an_indefinite_preconditioner(solver, cuda, cube5, precision):
    import torch

    b = _setup(solver, cube5, cuda, _abi.B2S_PRECOND_JACOBI, negate=True)
    x = torch.zeros_like(b)
    st = solver.pcg(b, x, tol=1e-6, stop_rule=_abi.B2S_STOP_RELRES, check_interval=1, precision=precision,
                    replace_every=50)
    assert st["bypassed"] == 1
    assert st["rz0"] > 0.0  # the plain start's r.r
    assert st["converged"] == 1 and st["rel_res"] <= 1e-6
    # the same arm in the oracle: bypassed too, and plain CG's iteration count
    A = O.OracleMatrix(cube5.n_verts, cube5.rows, cube5.cols, -cube5.vals)
    xo, info = O.pcg(A, -cube5.b, precond=O.ORC_PRECOND_JACOBI, tol=1e-6, stop_rule=O.ORC_STOP_RELRES)
    assert info["bypassed"] == 1 and info["converged"] == 1
    if precision == _abi.B2S_PRECISION_FP64:
        # plain CG over ~240 iterations: rounding (atomics in the SpMV) moves
        # the stop by a few iterations
        assert abs(st["iterations_exact"] - info["iterations"]) <= max(2, 0.05 * info["iterations"])
    # and, solved tightly, the solution is the unnegated system's
    x = torch.zeros_like(b)
    st = solver.pcg(b, x, tol=1e-11, stop_rule=_abi.B2S_STOP_RELRES, check_interval=5, precision=precision,
                    replace_every=50)
    assert st["bypassed"] == 1 and st["converged"] == 1
    A0 = O.OracleMatrix(cube5.n_verts, cube5.rows, cube5.cols, cube5.vals)
    xt, _, _ = O.cg_truth(A0, cube5.b, tol=1e-13)
    assert np.linalg.norm(x.cpu().numpy() - xt) <= 1e-6 * np.linalg.norm(xt)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_positive_definite_system_is_not_bypassed(solver, cuda, cube5, precision):
    import torch

    b = _setup(solver, cube5, cuda, _abi.B2S_PRECOND_MAS)
    x = torch.zeros_like(b)
    st = solver.pcg(b, x, tol=1e-4, stop_rule=_abi.B2S_STOP_RELRES, precision=precision)
    assert st["bypassed"] == 0 and st["converged"] == 1


@pytest.mark.parametrize("precision", PRECISIONS)
def test_nan_in_rhs_is_a_numeric_error(solver, cuda, cube5, precision):
    import torch

    b = _setup(solver, cube5, cuda, _abi.B2S_PRECOND_MAS)
    b[7] = float("nan")
    x = torch.zeros_like(b)
    with pytest.raises(B200SolveError) as ei:
        solver.pcg(b, x, tol=1e-4, stop_rule=_abi.B2S_STOP_RELRES, precision=precision)
    assert ei.value.code == _abi.B2S_ERR_NUMERIC
    # the handle stays usable: the next solve of a finite system works
    b[7] = 0.0
    st = solver.pcg(b, x, tol=1e-4, stop_rule=_abi.B2S_STOP_RELRES, precision=precision)
    assert st["converged"] == 1


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("use_graph", [True, False])
def test_iteration_cap_reports_not_converged(solver, cuda, cube5, precision, use_graph):
    import torch

    b = _setup(solver, cube5, cuda, _abi.B2S_PRECOND_JACOBI)
    x = torch.zeros_like(b)
    st = solver.pcg(b, x, tol=1e-10, stop_rule=_abi.B2S_STOP_RELRES, check_interval=1, max_iter=3,
                    precision=precision, use_graph=use_graph)
    assert st["converged"] == 0
    assert st["iterations"] == 3
    assert st["rel_res"] > 1e-10
    # x holds the third iterate (finite), and the solve can be resumed from it
    assert np.isfinite(x.cpu().numpy()).all() and np.isfinite(st["rel_res"])
    st2 = solver.pcg(b, x, tol=1e-6, stop_rule=_abi.B2S_STOP_RELRES, precision=precision, x0_given=True,
                     replace_every=50)
    assert st2["converged"] == 1 and st2["rel_res"] <= 1e-6


def test_warm_start_refused_by_its_check_is_zero(solver, cuda, cube5):
    """A start the FP64 check refuses falls back to x0 = 0: a history vector
    with a non-finite entry (its Galerkin coefficients are not finite), and
    random history vectors, which are kept only when the check passes."""
    import torch

    b = _setup(solver, cube5, cuda, _abi.B2S_PRECOND_MAS)
    solver.ws_init(hidden=64, seed=1)
    rng = np.random.default_rng(4)
    bad = to_dev(rng.standard_normal(3 * cube5.n_verts), cuda)
    bad[11] = float("inf")
    x0 = torch.full_like(b, 7.0)
    info = solver.ws_predict(b, x0, history=[bad], mode=_abi.B2S_WS_MODE_PREV)
    assert info["mode"] == _abi.B2S_WS_MODE_ZERO
    assert float(x0.abs().max()) == 0.0
    # random directions: either kept with a passing check, or zero
    junk = [to_dev(rng.standard_normal(3 * cube5.n_verts), cuda) for _ in range(3)]
    x1 = torch.full_like(b, 7.0)
    info = solver.ws_predict(b, x1, history=junk, mode=_abi.B2S_WS_MODE_HISTORY)
    if info["mode"] == _abi.B2S_WS_MODE_ZERO:
        assert float(x1.abs().max()) == 0.0
    else:
        assert info["rz_ratio"] < 1.0
    # and the PCG from the refused start is the plain solve
    st = solver.pcg(b, x0, tol=1e-4, stop_rule=_abi.B2S_STOP_RELRES, x0_given=True)
    xz = torch.zeros_like(b)
    st0 = solver.pcg(b, xz, tol=1e-4, stop_rule=_abi.B2S_STOP_RELRES)
    assert st["iterations_exact"] == st0["iterations_exact"]
