"""CPU checks of the synthetic cloth + affine-body system's block layout."""
import numpy as np


def test_cloth_abd_has_all_block_kinds():
    from libuipc_b200 import scene
    from oracle.oracle import OracleMatrix

    s = scene.cloth_on_bodies(24, 3, seed=3)
    off = 4 * s.n_bodies
    r, c = s.rows, s.cols
    body_body = (r < off) & (c < off)
    coupling = (r < off) & (c >= off)
    cloth = (r >= off) & (c >= off)
    assert s.n_contacts > 0
    # 16 per body (its 4 x 4 grid) + 10 per contact (the body's upper grid of the rank-1 contact term)
    assert body_body.sum() == 16 * s.n_bodies + 10 * s.n_contacts
    assert coupling.sum() == 4 * s.n_contacts and cloth.any()
    # the lower 3x3 blocks of each body's 4x4 grid are written as zeros
    low = body_body & (r > c)
    assert low.sum() == 6 * s.n_bodies and not s.vals[low].any()
    # symmetric positive definite
    A = OracleMatrix(s.n_verts, s.rows, s.cols, s.vals).to_scipy()
    assert abs(A - A.T).max() <= 1e-12 * abs(A).max()
    assert np.all(np.linalg.eigvalsh(A.toarray()) > 0)
