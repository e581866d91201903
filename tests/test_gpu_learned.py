"""Learned PCG warm start on the GPU: features, gradients and inference
against the CPU oracle (oracle/learned.py), and what the trained network
gains over the plain starts on a twisted-bar run."""
import numpy as np
import pytest

from libuipc_b200 import _abi
from oracle import learned as OL
from conftest import to_dev

pytestmark = pytest.mark.gpu

HIDDEN = 128


@pytest.fixture(scope="module")
def bar_system():
    from libuipc_b200 import scene

    return scene.twisted_bar(24, 4, 4, twist_deg=3.0, seed=2)


def _setup(solver, s, cuda):
    import torch

    from libuipc_b200.linear_system import partition_maps, partition_rcb

    p2r, r2p = partition_maps(partition_rcb(s.positions))
    solver.assemble(s.n_verts, to_dev(s.rows, cuda), to_dev(s.cols, cuda), to_dev(s.vals, cuda))
    solver.mas_init(0, s.n_verts, s.adj_start, s.adj_list, p2r, r2p)
    solver.precond_assemble(_abi.B2S_PRECOND_MAS)
    b = to_dev(s.b, cuda)
    z = torch.zeros_like(b)
    solver.precond_apply(b, z)
    beg, cnt, ct = solver.mas_hierarchy(s.n_verts)
    agg = ct[:, 0] - beg[1]
    agg[ct[:, 0] < 0] = -1
    return b, z, agg, int(cnt[1])


def test_features_match_oracle(solver, cuda, bar_system):
    s = bar_system
    b, z, agg, n_agg = _setup(solver, s, cuda)
    rng = np.random.default_rng(5)
    hist = [rng.standard_normal(3 * s.n_verts) * 1e-3 for _ in range(3)]
    x = rng.standard_normal(3 * s.n_verts) * 1e-3
    solver.ws_init(HIDDEN, seed=1)
    solver.ws_add_sample(b, to_dev(x, cuda), [to_dev(h, cuda) for h in hist])
    g = solver.ws_sample(0)
    ref = OL.aggregate(s.b, hist, z.cpu().numpy(), agg, n_agg, x)
    assert g["feat"].shape == ref["feat"].shape
    # FP32 atomics in arbitrary order: relative to each column's magnitude
    for key in ("feat", "H", "q"):
        err = np.abs(g[key] - ref[key]) / (np.abs(ref[key]).max(0, keepdims=True) + 1e-12)
        assert err.max() <= 1e-4, key
    assert np.allclose(g["c0"], ref["c0"], rtol=1e-4, atol=1e-6 * ref["c0"].max())
    assert g["norm"] == pytest.approx(ref["c0"].sum(), rel=1e-4)


def test_gradient_matches_oracle(solver, cuda, bar_system):
    """FP32 forward/backward kernels against the FP64 oracle on one sample,
    before and after a few training steps."""
    s = bar_system
    b, z, agg, n_agg = _setup(solver, s, cuda)
    rng = np.random.default_rng(6)
    hist = [rng.standard_normal(3 * s.n_verts) for _ in range(3)]
    x = hist[0] * 1.1 - 0.1 * hist[1] + 0.01 * rng.standard_normal(3 * s.n_verts)
    solver.ws_init(HIDDEN, seed=2)
    solver.ws_add_sample(b, to_dev(x, cuda), [to_dev(h, cuda) for h in hist])
    solver.ws_fit_normalization()
    for step in range(2):
        p = solver.ws_params()
        loss, grad = solver.ws_loss_grad(0)
        smp = solver.ws_sample(0)
        rl, rg, _ = OL.loss_grad(p.astype(np.float64), HIDDEN, smp)
        assert loss == pytest.approx(rl, rel=1e-4)
        assert np.linalg.norm(grad - rg) <= 1e-4 * np.linalg.norm(rg)
        solver.ws_train(3, lr=1e-3, seed=step)


def test_inference_matches_oracle(solver, cuda, bar_system):
    """BF16-weight inference + field + Galerkin scaling against the oracle's
    FP64 forward with the FP32 weights (no history: the field is c3 * z)."""
    import torch

    s = bar_system
    b, z, agg, n_agg = _setup(solver, s, cuda)
    solver.ws_init(HIDDEN, seed=3)
    p = solver.ws_params()
    L = OL.layout(HIDDEN)
    rng = np.random.default_rng(7)
    p[L["b2"]:L["n"]] += rng.standard_normal(OL.O).astype(np.float32)
    solver.ws_set_params(p)
    x0 = torch.zeros_like(b)
    info = solver.ws_predict(b, x0, [], _abi.B2S_WS_MODE_LEARNED)
    ref = OL.aggregate(s.b, [], z.cpu().numpy(), agg, n_agg)
    Y = OL.forward(p.astype(np.float64), HIDDEN, ref["feat"])
    zz = z.cpu().numpy().reshape(-1, 3)
    d = np.zeros_like(zz)
    keep = agg >= 0
    d[keep] = Y[agg[keep], 3][:, None] * zz[keep]
    d = d.ravel()
    from oracle.oracle import OracleMatrix

    A = OracleMatrix(s.n_verts, s.rows, s.cols, s.vals).to_scipy()
    alpha = d @ s.b / (d @ (A @ d))
    xr = alpha * d
    got = x0.cpu().numpy()
    if info["mode"] == _abi.B2S_WS_MODE_LEARNED:
        assert np.linalg.norm(got - xr) <= 2e-2 * np.linalg.norm(xr)
        r = s.b - A @ got
        assert info["rel_res0"] == pytest.approx(np.linalg.norm(r) / np.linalg.norm(s.b), rel=1e-6)
    else:
        # the check rejected the start: x0 = 0
        assert not got.any()
        assert info["rz_ratio"] >= 1.0


def test_mirror_pcg_with_history_start(solver, cuda):
    """B200PCG(warm_start='history') through GlobalLinearSystem over a run:
    once three earlier solutions exist the solves need far fewer iterations
    than the first one, and each still meets its stop rule."""
    from libuipc_b200.linear_system import B200MAS, B200PCG, GlobalLinearSystem, partition_maps, partition_rcb
    from libuipc_b200.sequence import SceneSequence

    seq = SceneSequence(scene=2, cells_x=30, cells_y=5, cells_z=5, E=1e6, nu=0.49, twist_per_step=2.0)
    p2r, r2p = partition_maps(partition_rcb(seq.rest))
    pre = B200MAS(0, seq.n_verts, seq.adj_start, seq.adj_list, p2r, r2p)
    pcg = B200PCG(tol_rate=1e-4, stop_rule=_abi.B2S_STOP_RELRES, warm_start="history")
    gls = GlobalLinearSystem(solver, pcg, pre)
    its = []

    def solve(sysm, step, k):
        dx = gls.solve(sysm.n_verts, to_dev(sysm.rows, cuda), to_dev(sysm.cols, cuda), to_dev(sysm.vals, cuda),
                       to_dev(sysm.b, cuda), history_slot=k)
        assert pcg.last_stats["rel_res"] <= 1e-4
        its.append(gls.last_solve_iterations)
        return -dx.cpu().numpy()

    for _ in seq.run(8, 1, solve):
        pass
    assert max(its[4:]) < 0.5 * its[0]


def test_learned_start_beats_plain_starts(solver, cuda):
    """Train on the first systems of a twisted-bar run, then solve the later
    ones (FP64-verified rel-res 1e-4) from each start: the trained network's
    start needs fewer PCG iterations than the zero and previous-dx starts."""
    from libuipc_b200.learned import SequenceRunner
    from libuipc_b200.sequence import SceneSequence

    seq = SceneSequence(scene=2, cells_x=40, cells_y=6, cells_z=6, E=1e6, nu=0.49, twist_per_step=2.0)
    run = SequenceRunner(solver, seq, cuda)
    solver.ws_init(HIDDEN, seed=0)
    run.run(16, newton_iters=1, collect=True)
    solver.ws_fit_normalization()
    loss = solver.ws_train(40, lr=1e-3, seed=0)
    assert np.isfinite(loss)
    log = run.run(8, newton_iters=1, collect=False, eval_modes=("zero", "prev", "history", "learned"))
    for r in log.records:
        assert r.rel_res <= 1e-4
    zero, prev = log.mean_iterations("zero"), log.mean_iterations("prev")
    hist, learned = log.mean_iterations("history"), log.mean_iterations("learned")
    print(f"mean PCG iterations: zero {zero:.1f} prev {prev:.1f} history {hist:.1f} learned {learned:.1f}")
    assert learned < 0.5 * zero
    assert learned < prev
    assert learned <= hist + 2


def test_longer_history_on_a_driven_bar(solver, cuda):
    """The Galerkin start over up to 8 past solutions (B2S_WS_MAX_HISTORY):
    on a smoothly driven run it needs no more PCG iterations than over the 3
    latest (here several times fewer), and a ninth history vector is refused."""
    import torch

    from libuipc_b200.learned import SequenceRunner
    from libuipc_b200.sequence import SceneSequence

    means = {}
    for keep in (3, 8):
        seq = SceneSequence(scene=2, cells_x=40, cells_y=6, cells_z=6, E=1e6, nu=0.49, twist_per_step=2.0)
        run = SequenceRunner(solver, seq, cuda, history=keep)
        run.run(10, newton_iters=1, collect=False)
        log = run.run(6, newton_iters=1, collect=False, eval_modes=("history",))
        assert all(r.rel_res <= 1e-4 for r in log.records)
        means[keep] = log.mean_iterations("history")
        if keep == 8:
            assert len(run.hist(0)) == 8
            import ctypes as C

            from libuipc_b200 import _abi

            b = torch.ones(3 * seq.n_verts, dtype=torch.float64, device=cuda)
            x = torch.zeros_like(b)
            nine = run.hist(0) + [b]
            arr = (C.c_void_p * 9)(*[h.data_ptr() for h in nine])
            info = _abi.WsInfo()
            rc = solver.lib.b2s_ws_predict(solver.h, _abi.B2S_WS_MODE_HISTORY, C.c_void_p(b.data_ptr()), 9,
                                           C.cast(arr, C.c_void_p), C.c_void_p(x.data_ptr()), C.byref(info))
            assert rc == _abi.B2S_ERR_ARGUMENT
            assert b"history length" in solver.lib.b2s_last_error(solver.h)
            # the Python wrapper keeps the newest 8
            assert solver.ws_predict(b, x, nine, _abi.B2S_WS_MODE_HISTORY)["n_candidates"] <= 8
    print(f"history start: 3 latest {means[3]:.1f}, 8 latest {means[8]:.1f} PCG iterations")
    assert means[8] <= means[3]


def test_checkpoint_round_trip(solver, cuda, tmp_path):
    """save_checkpoint / load_checkpoint: a second solver restored from the
    file holds the same parameters and training set, so its loss and
    gradient on every stored sample are the first solver's, and so is its
    prediction on the same system (up to the order of atomic sums in the
    feature reductions)."""
    import torch

    from libuipc_b200.learned import SequenceRunner, load_checkpoint, save_checkpoint
    from libuipc_b200.linear_system import Solver
    from libuipc_b200.sequence import SceneSequence

    seq = SceneSequence(scene=2, cells_x=24, cells_y=4, cells_z=4, E=1e6, nu=0.49, twist_per_step=2.0)
    run = SequenceRunner(solver, seq, cuda)
    solver.ws_init(64, seed=3)
    run.run(6, newton_iters=1, collect=True)
    solver.ws_fit_normalization()
    solver.ws_train(3, lr=1e-3, seed=0)
    path = str(tmp_path / "ws.npz")
    save_checkpoint(solver, path)
    n, rows = solver.ws_num_samples()
    assert n >= 3

    other = Solver(0)
    try:
        assert load_checkpoint(other, path) == n
        assert other.ws_num_samples() == (n, rows)
        assert np.array_equal(other.ws_params(), solver.ws_params())
        for i in range(n):
            a, b = solver.ws_sample(i), other.ws_sample(i)
            for k in ("feat", "H", "q", "c0"):
                assert np.array_equal(a[k], b[k]), (i, k)
            assert a["norm"] == b["norm"]
            la, ga = solver.ws_loss_grad(i)
            lb, gb = other.ws_loss_grad(i)
            assert abs(la - lb) <= 1e-6 * abs(la)
            assert np.abs(ga - gb).max() <= 1e-5 * np.abs(ga).max()
        # the same prediction on the same system and history
        sysm = seq.system()
        hist = run.hist(0)
        for sv in (solver, other):
            _setup(sv, sysm, cuda)
        b = to_dev(sysm.b, cuda)
        xa, xb = torch.zeros_like(b), torch.zeros_like(b)
        ia = solver.ws_predict(b, xa, history=hist)
        ib = other.ws_predict(b, xb, history=hist)
        assert ia["mode"] == ib["mode"]
        assert float((xa - xb).norm()) <= 1e-7 * float(xa.norm())  # FP32 feature sums
    finally:
        other.close()
    # a file of another format version is refused
    d = dict(np.load(path))
    d["version"] = np.int32(99)
    np.savez(str(tmp_path / "bad.npz"), **d)
    with pytest.raises(ValueError):
        load_checkpoint(solver, str(tmp_path / "bad.npz"))
