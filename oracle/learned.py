"""CPU restatement of the learned PCG warm start (test infrastructure only).

Checks the CUDA implementation in libuipc_b200/csrc/b2s_learned.cu: the
per-aggregate features and training statistics, and the MLP loss and its
gradient, in FP64 with numpy. Nothing in the product imports this module.
The learned warm start has no counterpart in the reference (its PCG starts
from zero, src/backends/cuda/linear_system/linear_fused_pcg.cu:1782-2005), so
there is nothing of the reference to pin it to: the checks are
self-consistency of GPU against this restatement.
"""
from __future__ import annotations

import numpy as np

F = 22  # features
O = 4  # outputs = fields
NF = 4


def layout(hidden: int) -> dict:
    """Offsets of W0[F x H] b0[H] W1[H x H] b1[H] W2[H x O] b2[O]."""
    H = hidden
    o = {}
    o["W0"] = 0
    o["b0"] = o["W0"] + F * H
    o["W1"] = o["b0"] + H
    o["b1"] = o["W1"] + H * H
    o["W2"] = o["b1"] + H
    o["b2"] = o["W2"] + H * O
    o["n"] = o["b2"] + O
    return o


def unpack(params: np.ndarray, hidden: int):
    L = layout(hidden)
    H = hidden
    p = params.astype(np.float64)
    W0 = p[L["W0"]:L["b0"]].reshape(F, H)
    b0 = p[L["b0"]:L["W1"]]
    W1 = p[L["W1"]:L["b1"]].reshape(H, H)
    b1 = p[L["b1"]:L["W2"]]
    W2 = p[L["W2"]:L["b2"]].reshape(H, O)
    b2 = p[L["b2"]:L["n"]]
    mean = p[L["n"]:L["n"] + F]
    std = p[L["n"] + F:L["n"] + 2 * F]
    return W0, b0, W1, b1, W2, b2, mean, std


def fields(b, hist, z):
    """f0 = h1, f1 = h1 - h2, f2 = h1 - 2 h2 + h3, f3 = z (missing history = 0)."""
    h = [np.asarray(v, np.float64) for v in hist] + [np.zeros_like(b)] * (3 - len(hist))
    return [h[0], h[0] - h[1], h[0] - 2 * h[1] + h[2], np.asarray(z, np.float64)]


def aggregate(b, hist, z, agg, n_agg, x=None):
    """Features [n_agg, 22] and (with x) the Gram H (upper, 10), q (4), c0 of
    every aggregate; agg[v] = level-1 aggregate of vertex v (-1 = none)."""
    b = np.asarray(b, np.float64)
    n = b.size
    f = fields(b, hist, z)
    sz = np.sqrt(np.dot(f[3], f[3]) / n) or 1.0
    sb = np.sqrt(np.dot(b, b) / n) or 1.0
    keep = agg >= 0
    a = agg[keep]
    B = b.reshape(-1, 3)[keep] / sb
    Fv = [fi.reshape(-1, 3)[keep] / sz for fi in f]

    def s(w):
        return np.bincount(a, w, minlength=n_agg)

    cnt = np.maximum(s(np.ones(a.size)), 1.0)
    feats = [s(B[:, c]) / cnt for c in range(3)]
    for fi in Fv:
        feats += [s(fi[:, c]) / cnt for c in range(3)]
        feats.append(np.log(np.sqrt(np.maximum(s((fi * fi).sum(1)), 0) / cnt) + 1e-6))
    for i in range(NF - 1):
        feats.append(s((Fv[i] * Fv[i + 1]).sum(1)) / cnt)
    out = {"feat": np.stack(feats, 1)}
    if x is not None:
        X = np.asarray(x, np.float64).reshape(-1, 3)[keep] / sz
        Hs = [s((Fv[i] * Fv[j]).sum(1)) for i in range(NF) for j in range(i, NF)]
        out["H"] = np.stack(Hs, 1)
        out["q"] = np.stack([s((Fv[i] * X).sum(1)) for i in range(NF)], 1)
        out["c0"] = s((X * X).sum(1))
    return out


def sym(Hs: np.ndarray) -> np.ndarray:
    """[rows, 10] upper triangle -> [rows, 4, 4]."""
    r = Hs.shape[0]
    M = np.zeros((r, NF, NF))
    e = 0
    for i in range(NF):
        for j in range(i, NF):
            M[:, i, j] = M[:, j, i] = Hs[:, e]
            e += 1
    return M


def loss_grad(params: np.ndarray, hidden: int, sample: dict):
    """Loss sum_a (y^T H y - 2 y^T q + c0) / norm and its gradient w.r.t. the
    network parameters (same layout as the device vector, without the
    standardisation entries)."""
    W0, b0, W1, b1, W2, b2, mean, std = unpack(params, hidden)
    X = (sample["feat"].astype(np.float64) - mean) / np.maximum(std, 1e-3)
    Hm = sym(sample["H"].astype(np.float64))
    q = sample["q"].astype(np.float64)
    c0 = sample["c0"].astype(np.float64)
    norm = sample["norm"]
    Z1 = X @ W0 + b0
    H1 = np.maximum(Z1, 0)
    Z2 = H1 @ W1 + b1
    H2 = np.maximum(Z2, 0)
    Y = H2 @ W2 + b2
    Hy = np.einsum("aij,aj->ai", Hm, Y)
    loss = ((Y * Hy).sum(1) - 2 * (Y * q).sum(1) + c0).sum() / norm
    dY = 2 * (Hy - q) / norm
    gW2 = H2.T @ dY
    gb2 = dY.sum(0)
    dH2 = (dY @ W2.T) * (H2 > 0)
    gW1 = H1.T @ dH2
    gb1 = dH2.sum(0)
    dH1 = (dH2 @ W1.T) * (H1 > 0)
    gW0 = X.T @ dH1
    gb0 = dH1.sum(0)
    g = np.concatenate([gW0.ravel(), gb0, gW1.ravel(), gb1, gW2.ravel(), gb2])
    return loss, g, Y


def forward(params: np.ndarray, hidden: int, feat: np.ndarray) -> np.ndarray:
    W0, b0, W1, b1, W2, b2, mean, std = unpack(params, hidden)
    X = (feat.astype(np.float64) - mean) / np.maximum(std, 1e-3)
    H1 = np.maximum(X @ W0 + b0, 0)
    H2 = np.maximum(H1 @ W1 + b1, 0)
    return H2 @ W2 + b2
