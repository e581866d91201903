"""CPU checks of the learned warm start's host side: the oracle's MLP
gradient against finite differences, the oracle's aggregation against a
direct loop, and the scene stepping used to generate training systems."""
import numpy as np
import pytest

from oracle import learned as OL


def _sample(rng, rows=37):
    # a PSD Gram per row, as the field Gram is
    F = rng.standard_normal((rows, 6, OL.NF))
    G = np.einsum("rki,rkj->rij", F, F)
    iu = np.triu_indices(OL.NF)
    x = rng.standard_normal((rows, 6))
    q = np.einsum("rki,rk->ri", F, x)
    return {"feat": rng.standard_normal((rows, OL.F)), "H": G[:, iu[0], iu[1]], "q": q,
            "c0": (x * x).sum(1), "norm": float((x * x).sum())}


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    hidden = 64
    L = OL.layout(hidden)
    p = rng.standard_normal(L["n"] + 2 * OL.F) * 0.2
    p[L["n"]:L["n"] + OL.F] = rng.standard_normal(OL.F) * 0.1  # mean
    p[L["n"] + OL.F:] = 0.5 + rng.random(OL.F)  # std
    smp = _sample(rng)
    loss, g, _ = OL.loss_grad(p, hidden, smp)
    for idx in rng.choice(L["n"], 25, replace=False):
        e = np.zeros_like(p)
        e[idx] = 1e-6
        fd = (OL.loss_grad(p + e, hidden, smp)[0] - OL.loss_grad(p - e, hidden, smp)[0]) / 2e-6
        assert abs(fd - g[idx]) <= 1e-6 * max(1.0, abs(fd)), idx


def test_oracle_loss_is_field_error():
    """The quadratic loss equals sum |d - x|^2 / sum |x|^2 of the field it
    describes (here built directly)."""
    rng = np.random.default_rng(4)
    nv, n_agg = 60, 7
    agg = rng.integers(-1, n_agg, nv)
    agg[:n_agg] = np.arange(n_agg)
    b = rng.standard_normal(3 * nv)
    hist = [rng.standard_normal(3 * nv) for _ in range(3)]
    z = rng.standard_normal(3 * nv)
    x = rng.standard_normal(3 * nv)
    s = OL.aggregate(b, hist, z, agg, n_agg, x)
    y = rng.standard_normal((n_agg, OL.NF))
    Hm = OL.sym(s["H"])
    quad = (np.einsum("ai,aij,aj->a", y, Hm, y) - 2 * (y * s["q"]).sum(1) + s["c0"]).sum()
    f = OL.fields(b, hist, z)
    sz = np.sqrt(np.dot(z, z) / z.size)
    keep = agg >= 0
    d = sum(y[agg[keep], i][:, None] * f[i].reshape(-1, 3)[keep] for i in range(OL.NF)) / sz
    X = x.reshape(-1, 3)[keep] / sz
    assert quad == pytest.approx(((d - X) ** 2).sum(), rel=1e-10)


def test_generate_state_reproduces_default_system():
    from libuipc_b200 import scene

    for cfg in (dict(scene=2, cells_x=8, cells_y=3, cells_z=3, twist_deg=0.0),
                dict(scene=1, cells_x=4, cells_y=4, cells_z=4, n_cubes=2)):
        s0 = scene.generate(**cfg)
        c = s0.config
        xt = s0.positions.copy()
        xt[:, 1] -= c["dt"] ** 2 * c["gravity"]
        s1 = scene.generate_state(s0.positions, xt, **cfg)
        assert np.array_equal(s0.rows, s1.rows) and np.array_equal(s0.cols, s1.cols)
        assert np.array_equal(s0.vals, s1.vals)
        assert np.allclose(s0.b, s1.b, rtol=0, atol=1e-18)


def test_sequence_twist_moves_only_the_ends_first():
    from libuipc_b200.sequence import SceneSequence

    seq = SceneSequence(scene=2, cells_x=8, cells_y=3, cells_z=3, twist_per_step=5.0)
    seq.begin_step()
    moved = np.abs(seq.x - seq.rest).max(1) > 0
    assert np.array_equal(moved, seq.fixed)
    sysm = seq.system()
    # fixed rows: identity diagonal, zero gradient
    assert np.allclose(sysm.b.reshape(-1, 3)[seq.fixed], 0)


def test_checkpoint_width_from_parameter_count():
    """The hidden width a checkpoint records is recovered from the parameter
    count b2s_ws_get_params reports (weights, biases and 2 x 22 statistics)."""
    from libuipc_b200 import _abi
    from libuipc_b200.learned import _hidden_of

    F, O = _abi.B2S_WS_FEATURES, _abi.B2S_WS_OUTPUTS
    for h in (64, 128, 256, 512):
        n = F * h + h + h * h + h + h * O + O + 2 * F
        assert _hidden_of(n) == h
    with pytest.raises(ValueError):
        _hidden_of(1000)
