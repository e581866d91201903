"""The GPU Newton-system generator (include/b200gen.h) against the host
generator (csrc/scene/scene_gen.cpp): the same block pattern after assembly,
values and gradient to rounding (the device contracts multiply-adds; relative
1e-11 of the largest entry), on a twisted bar at a deformed state (Dirichlet
ends) and on a cube on the ground (barrier blocks)."""
import numpy as np
import pytest

from conftest import to_dev

pytestmark = pytest.mark.gpu


def _assembled(solver, nb, rows, cols, vals):
    solver.assemble(nb, rows, cols, vals)
    return solver.upper_bsr()


def _compare(solver, cuda, s_cpu, gen_out):
    rows, cols, vals, b = gen_out
    rp1, c1, v1 = _assembled(solver, s_cpu.n_verts, to_dev(s_cpu.rows, cuda), to_dev(s_cpu.cols, cuda),
                             to_dev(s_cpu.vals, cuda))
    rp2, c2, v2 = _assembled(solver, s_cpu.n_verts, rows, cols, vals)
    assert np.array_equal(rp1, rp2) and np.array_equal(c1, c2)
    scale = np.abs(v1).max()
    assert np.abs(v1 - v2).max() <= 1e-11 * scale
    bg = b.cpu().numpy()
    assert np.abs(bg - s_cpu.b).max() <= 1e-11 * np.abs(s_cpu.b).max()


def test_twisted_bar_state(solver, cuda):
    import torch

    from libuipc_b200 import scene
    from libuipc_b200.gpu_scene import GpuTetMesh
    from libuipc_b200.sequence import SceneSequence

    seq = SceneSequence(scene=2, cells_x=20, cells_y=4, cells_z=4, E=1e6, nu=0.49, twist_per_step=3.0)
    seq.begin_step()
    s_cpu = seq.system()
    mesh = GpuTetMesh(seq.rest, s_cpu.tets, s_cpu.config, cuda, fixed=seq.fixed)
    try:
        x = to_dev(seq.x.ravel(), cuda)
        xt = to_dev(seq.x_tilde.ravel(), cuda)
        _compare(solver, cuda, s_cpu, mesh.system(x, xt))
    finally:
        mesh.close()


def test_cube_on_ground(solver, cuda):
    from libuipc_b200 import scene
    from libuipc_b200.gpu_scene import GpuTetMesh

    s_cpu = scene.cube_on_ground(6, seed=2)
    c = s_cpu.config
    vx = vy = 7
    v = np.arange(s_cpu.n_verts)
    bottom = v[(v // vx) % vy == 0].astype(np.int32)
    ground_y = s_cpu.positions[bottom, 1].min() - c["ground_offset"]
    mesh = GpuTetMesh(s_cpu.positions, s_cpu.tets, c, cuda, ground=bottom, ground_y=ground_y)
    try:
        x = to_dev(s_cpu.positions.ravel(), cuda)
        xt = s_cpu.positions.copy()
        xt[:, 1] -= c["dt"] ** 2 * c["gravity"]
        _compare(solver, cuda, s_cpu, mesh.system(x, to_dev(xt.ravel(), cuda)))
    finally:
        mesh.close()


def test_generator_writes_into_solver_owned_triplets(solver, cuda):
    """b2s_triplet_buffers + b2s_assemble_owned: the producer writes in place
    (no staging copy) and the assembled matrix is the same."""
    from libuipc_b200.gpu_scene import GpuTetMesh
    from libuipc_b200.sequence import SceneSequence

    seq = SceneSequence(scene=2, cells_x=12, cells_y=3, cells_z=3, E=1e6, nu=0.49, twist_per_step=2.0)
    seq.begin_step()
    s = seq.system()
    mesh = GpuTetMesh(seq.rest, s.tets, s.config, cuda, fixed=seq.fixed)
    try:
        x, xt = to_dev(seq.x.ravel(), cuda), to_dev(seq.x_tilde.ravel(), cuda)
        rows, cols, vals, _ = mesh.system(x, xt)
        solver.assemble(s.n_verts, rows, cols, vals)
        ref = solver.upper_bsr()
        r_ptr, c_ptr, v_ptr = solver.triplet_buffers(mesh.n_triplets)
        mesh.system_into(x, xt, r_ptr, c_ptr, v_ptr)
        solver.assemble_owned(s.n_verts, mesh.n_triplets)
        got = solver.upper_bsr()
        assert all(np.array_equal(a, b) for a, b in zip(ref, got))
        with pytest.raises(RuntimeError):
            solver.assemble_owned(s.n_verts, mesh.n_triplets * 2)  # more than the buffers hold
    finally:
        mesh.close()


def _grid_tris(N):
    t = []
    for k in range(N - 1):
        for i in range(N - 1):
            a, b, c, d = i + N * k, i + 1 + N * k, i + 1 + N * (k + 1), i + N * (k + 1)
            t += [(a, b, c), (a, c, d)]
    return np.array(t, np.int32)


def test_cloth_producers_match_the_host_generator(cuda):
    """The cloth of the cloth-over-bodies scene (48 x 48 vertices, 16 bodies)
    from the device producers (kinetic, Baraff-Witkin, discrete-shell
    bending) against the host generator's triplets in the same slots, and the
    gradient on the vertices no contact touches."""
    import torch

    from libuipc_b200 import scene
    from libuipc_b200.gpu_scene import GpuShell

    N, dt, g = 48, 0.01, 9.8
    s = scene.cloth_on_bodies(N, 4, seed=0)
    nb = s.n_bodies
    off = 4 * nb
    hc = 2.0 / (N - 1)
    mass = np.full(N * N, 1e3 * 1e-3 * hc * hc)
    rest = s.positions[off:]  # first step from rest: x = rest
    sh = GpuShell(rest, _grid_tris(N), mass, stretch=1e3, shear=1e2, bend=1e-2, dt=dt, device=cuda)
    T = sh.n_triplets
    assert sh.n_hinges == 3 * (N - 1) ** 2 - 2 * (N - 1)
    x = to_dev(s.positions.reshape(-1), cuda)
    xt = x.clone()
    xt[1::3] -= dt * dt * g
    rows = torch.empty(T, dtype=torch.int32, device=cuda)
    cols = torch.empty_like(rows)
    vals = torch.empty((T, 9), dtype=torch.float64, device=cuda)
    grad = torch.zeros(3 * s.n_verts, dtype=torch.float64, device=cuda)
    sh.system_into(x, xt, off, rows.data_ptr(), cols.data_ptr(), vals.data_ptr(), grad)
    h0 = 16 * nb
    assert np.array_equal(rows.cpu().numpy(), s.rows[h0:h0 + T])
    assert np.array_equal(cols.cpu().numpy(), s.cols[h0:h0 + T])
    hv = s.vals[h0:h0 + T]
    assert np.abs(vals.cpu().numpy() - hv).max() <= 1e-11 * np.abs(hv).max()
    touched = np.unique(np.concatenate([s.rows[h0 + T:], s.cols[h0 + T:]]))
    keep = np.setdiff1d(np.arange(off, s.n_verts), touched)
    assert keep.size > N * N // 2
    gd = grad.cpu().numpy().reshape(-1, 3)[keep]
    gh = s.b.reshape(-1, 3)[keep]
    assert np.abs(gd - gh).max() <= 1e-11 * np.abs(gh).max()
    sh.close()


def test_affine_body_producer_against_the_oracle(cuda):
    """Kinetic + orthogonality potential of 7 affine bodies at random states
    (near-rotations and general affine matrices) against the oracle's
    restatement (mass matrix + PSD part of the finite-difference Hessian)."""
    import torch

    from libuipc_b200.gpu_scene import GpuAffineBodies
    from oracle import elements as OE

    rng = np.random.default_rng(7)
    nb, dt, kappa = 7, 0.01, 1e8
    M = np.zeros((nb, 12, 12))
    q = np.zeros((nb, 12))
    for b in range(nb):
        m, I = rng.uniform(0.5, 2.0), rng.uniform(0.01, 0.1)
        M[b] = np.diag([m] * 3 + [I] * 9)
        R, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        A = R + (0.05 if b % 2 else 0.5) * rng.standard_normal((3, 3))
        q[b] = np.concatenate([rng.standard_normal(3), A.T.reshape(-1)])
    vol = rng.uniform(1e-4, 1e-3, nb)
    qt = q + 1e-3 * rng.standard_normal(q.shape)
    ab = GpuAffineBodies(M, np.full(nb, kappa), vol, dt, cuda)
    T = 16 * nb
    rows = torch.empty(T, dtype=torch.int32, device=cuda)
    cols = torch.empty_like(rows)
    vals = torch.empty((T, 9), dtype=torch.float64, device=cuda)
    grad = torch.zeros(12 * nb, dtype=torch.float64, device=cuda)
    ab.system_into(to_dev(q.reshape(-1), cuda), to_dev(qt.reshape(-1), cuda), 0, rows.data_ptr(), cols.data_ptr(),
                   vals.data_ptr(), grad)
    V = vals.cpu().numpy().reshape(nb, 4, 4, 3, 3)  # [b, bi, bj, col, row]
    G = grad.cpu().numpy().reshape(nb, 12)
    for b in range(nb):
        _, Go, Ho = OE.ortho_element(q[b], kappa, vol[b] * dt * dt)
        H = M[b].copy()
        H[3:, 3:] += Ho
        for bi in range(4):
            for bj in range(4):
                blk = V[b, bi, bj].T
                ref = H[3 * bi:3 * bi + 3, 3 * bj:3 * bj + 3] if bi <= bj else np.zeros((3, 3))
                assert np.abs(blk - ref).max() <= 1e-5 * np.abs(H).max(), (b, bi, bj)
        Gr = M[b] @ (q[b] - qt[b])
        Gr[3:] += Go
        assert np.abs(G[b] - Gr).max() <= 1e-6 * np.abs(Gr).max() + 1e-10 * kappa * vol[b] * dt * dt
    r = rows.cpu().numpy().reshape(nb, 4, 4)
    c = cols.cpu().numpy().reshape(nb, 4, 4)
    for b in range(nb):
        assert np.array_equal(r[b], 4 * b + np.arange(4)[:, None].repeat(4, 1))
        assert np.array_equal(c[b], 4 * b + np.arange(4)[None, :].repeat(4, 0))
    ab.close()


def test_contact_producer_against_the_host_routines(cuda):
    """Point-triangle, edge-edge, point-edge, point-point and near-parallel
    (mollified) pairs on the device against the host build of the same
    element routine (b2g_element_contact), which the CPU tests check against
    the oracle: every block to 1e-8 of the pair's largest entry (the PSD
    projection's Jacobi sweeps meet FMA-contracted inputs), and the gradient
    sums per vertex in pair order."""
    import ctypes as C
    import sys
    import os

    import torch

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_elements_cpu import _contact_case, _lib_contact

    from libuipc_b200.gpu_scene import GpuContacts

    rng = np.random.default_rng(11)
    dhat, kappa, dt = 1e-3, 1e9, 0.01
    X, pairs, is_ee, eps = [], [], [], []
    for i, kind in enumerate(["PT", "PE", "PP", "EE", "EE-parallel"] * 6):
        Xi, ee = _contact_case(kind, rng, dhat)
        X.append(Xi)
        pairs.append([4 * i, 4 * i + 1, 4 * i + 2, 4 * i + 3])
        is_ee.append(ee)
        ea, eb = Xi[1] - Xi[0], Xi[3] - Xi[2]
        eps.append(1e-3 * (ea @ ea) * (eb @ eb))
    # a shared vertex: the last pair reuses vertex 0 of the first
    pairs[-1][0] = 0
    X[-1][0] = X[0][0]
    Xall = np.concatenate(X)
    n = len(pairs)
    gc = GpuContacts(np.array(pairs), np.array(is_ee), np.array(eps), dhat, kappa, dt, cuda)
    rows = torch.empty(10 * n, dtype=torch.int32, device=cuda)
    cols = torch.empty_like(rows)
    vals = torch.empty((10 * n, 9), dtype=torch.float64, device=cuda)
    grad = torch.zeros(Xall.size, dtype=torch.float64, device=cuda)
    gc.system_into(to_dev(Xall.reshape(-1), cuda), rows.data_ptr(), cols.data_ptr(), vals.data_ptr(), grad)
    V = vals.cpu().numpy().reshape(n, 10, 3, 3)
    types = gc.types()
    gref = np.zeros_like(Xall.reshape(-1))
    for p in range(n):
        Xp = Xall[pairs[p]]
        t, G, H = _lib_contact(Xp, is_ee[p], eps[p], dhat, kappa * dt * dt)
        assert types[p] == t, (p, int(types[p]), t)
        scale = max(np.abs(H).max(), 1e-300)
        k = 0
        for i in range(4):
            for j in range(i, 4):
                a, b = pairs[p][i], pairs[p][j]
                blk = H[3 * i:3 * i + 3, 3 * j:3 * j + 3]
                ref = blk if a <= b else blk.T
                assert np.abs(V[p, k].T - ref).max() <= 1e-8 * scale, (p, i, j)
                k += 1
        for i in range(4):
            gref[3 * pairs[p][i]:3 * pairs[p][i] + 3] += G[3 * i:3 * i + 3]
    assert np.abs(grad.cpu().numpy() - gref).max() <= 1e-10 * np.abs(gref).max()
    gc.close()
