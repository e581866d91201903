"""The contact term of the line search on the device (b2gen_contacts_energy,
b2gen_contacts_toi): the pairs' barrier energy and the trajectory filter's
step bound (swept-AABB test, then additive CCD) against the oracle's
restatement (oracle/elements.py: contact_energy, pairs_toi) on random
point-triangle / edge-edge pairs, an analytic time of impact, and a line
search on two stacked cubes whose step the contact pairs cut: no pair
crosses, and the accepted state is the oracle's."""
import numpy as np
import pytest

from conftest import to_dev

pytestmark = pytest.mark.gpu


def _random_pairs(n, seed):
    """n pairs with their own 4 vertices each: a point above a triangle
    (point-triangle) or two crossing edges one above the other (edge-edge),
    gaps from 1e-5 to 2e-3, moving towards each other by up to 3x the gap
    with some sideways motion."""
    rng = np.random.default_rng(seed)
    X, D, P, E = [], [], [], []
    for i in range(n):
        ee = i % 2 == 1
        h = 10 ** rng.uniform(-5, np.log10(2e-3))
        if ee:
            a0 = np.array([-1.0, 0.0, 0.0]) * 0.01 + 0.002 * rng.standard_normal(3)
            a1 = np.array([1.0, 0.0, 0.0]) * 0.01 + 0.002 * rng.standard_normal(3)
            b0 = np.array([0.0, 0.0, -1.0]) * 0.01 + 0.002 * rng.standard_normal(3)
            b1 = np.array([0.0, 0.0, 1.0]) * 0.01 + 0.002 * rng.standard_normal(3)
            b0[1] = b1[1] = max(a0[1], a1[1]) + h + 0.004
            x4 = np.stack([a0, a1, b0, b1])
            d4 = np.zeros((4, 3))
            d4[2:, 1] = -rng.uniform(0.0, 3.0) * (h + 0.004)
        else:
            t = 0.01 * rng.standard_normal((3, 3))
            t[:, 1] = 0.001 * rng.standard_normal(3)
            c = t.mean(0)
            p = c + np.array([0.0, h + abs(t[:, 1]).max(), 0.0])
            x4 = np.vstack([p, t])
            d4 = np.zeros((4, 3))
            d4[0, 1] = -rng.uniform(0.0, 3.0) * (p[1] - t[:, 1].min())
        d4 += 1e-4 * rng.standard_normal((4, 3))
        base = 4 * i
        X.append(x4)
        D.append(d4)
        P.append([base, base + 1, base + 2, base + 3])
        E.append(1 if ee else 0)
    return np.vstack(X), np.vstack(D), np.array(P, np.int32), np.array(E, np.uint8)


def test_energy_and_toi_match_the_oracle(cuda):
    from libuipc_b200.gpu_scene import GpuContacts
    from oracle import elements as OE

    x, d, pairs, is_ee = _random_pairs(512, seed=3)
    dhat, kappa, dt = 5e-3, 1e6, 1e-2
    eps = np.full(len(pairs), 1e-3 * 4e-4 * 4e-4)
    C = GpuContacts(pairs, is_ee, eps, dhat, kappa, dt, cuda)
    try:
        k = kappa * dt * dt
        e_ref = sum(OE.contact_energy(x[p], ee, ep, dhat, k) for p, ee, ep in zip(pairs, is_ee, eps))
        e_dev = C.energy(to_dev(x.ravel(), cuda))
        assert e_ref > 0 and abs(e_dev - e_ref) <= 1e-12 * abs(e_ref)
        for alpha in (1.0, 0.5):
            t_ref = OE.pairs_toi(x, d, pairs, is_ee, alpha, dhat)
            t_dev = C.toi(to_dev(x.ravel(), cuda), to_dev(d.ravel(), cuda), alpha=alpha)
            assert t_ref < 1.0 and abs(t_dev - t_ref) <= 1e-9 * t_ref
        # per pair: the one pair alone gives its own time of impact
        for i in (0, 1, 2, 3):
            Ci = GpuContacts(pairs[i:i + 1] - 4 * i, is_ee[i:i + 1], eps[i:i + 1], dhat, kappa, dt, cuda)
            try:
                xi, di = x[4 * i:4 * i + 4], d[4 * i:4 * i + 4]
                t_ref = OE.pairs_toi(xi, di, [[0, 1, 2, 3]], is_ee[i:i + 1], 1.0, dhat)
                t_dev = Ci.toi(to_dev(xi.ravel(), cuda), to_dev(di.ravel(), cuda))
                assert abs(t_dev - t_ref) <= 1e-9 * t_ref
            finally:
                Ci.close()
    finally:
        C.close()


def test_analytic_time_of_impact_and_no_motion(cuda):
    """A point 1 mm above a triangle moving 2 mm straight down: the first
    advance covers (1 - eta) of the distance and the next one falls below
    eta of it, so the time of impact is (1 - eta) / 2 = 0.45; parallel
    motion of the whole pair (no relative displacement) gives no impact."""
    from libuipc_b200.gpu_scene import GpuContacts

    x = np.array([[0.2e-2, 1e-3, 0.2e-2], [0.0, 0.0, 0.0], [1e-2, 0.0, 0.0], [0.0, 0.0, 1e-2]])
    d = np.zeros((4, 3))
    d[0, 1] = -2e-3
    C = GpuContacts(np.array([[0, 1, 2, 3]], np.int32), np.array([0], np.uint8), np.array([0.0]), 2e-3, 1e6, 1e-2,
                    cuda)
    try:
        assert abs(C.toi(to_dev(x.ravel(), cuda), to_dev(d.ravel(), cuda)) - 0.45) <= 1e-12
        d[:] = -2e-3
        assert C.toi(to_dev(x.ravel(), cuda), to_dev(d.ravel(), cuda)) == 1.0
        assert C.energy(to_dev(x.ravel(), cuda)) > 0.0
    finally:
        C.close()


def _two_cubes(cuda, cells=4, lift=2e-3):
    from libuipc_b200 import scene
    from libuipc_b200.gpu_scene import GpuTetMesh

    s = scene.cube_on_ground(cells, seed=2)
    c = dict(s.config)
    n, v, vx = s.n_verts, np.arange(s.n_verts), cells + 1
    P = s.positions
    height = P[:, 1].max() - P[:, 1].min()
    up = P + np.array([0.0, height + lift, 0.0])
    pos = np.vstack([P, up])
    tets = np.vstack([s.tets, s.tets + n])
    iy, ix, iz = (v // vx) % vx, v % vx, v // (vx * vx)
    top = v[iy == cells]
    bottom_up = v[iy == 0] + n
    ground = v[iy == 0].astype(np.int32)
    ground_y = P[ground, 1].min() - c["ground_offset"]
    # top-face triangles of the lower cube (two per grid quad) and edges of
    # the faces that meet
    idx = {(int(ix[t]), int(iz[t])): int(t) for t in top}
    tris, top_edges, bot_edges = [], [], []
    for i in range(cells):
        for k in range(cells):
            a, b, cc, dd = idx[(i, k)], idx[(i + 1, k)], idx[(i + 1, k + 1)], idx[(i, k + 1)]
            tris += [(a, b, cc), (a, cc, dd)]
    for (i, k), t in idx.items():
        for di, dk in ((1, 0), (0, 1)):
            if (i + di, k + dk) in idx:
                top_edges.append((t, idx[(i + di, k + dk)]))
                bot_edges.append((t + n - (cells) * vx, idx[(i + di, k + dk)] + n - cells * vx))
    pairs, is_ee = [], []
    h = np.ptp(P[:, 0]) / cells
    for p in bottom_up:
        for tri in tris:
            cxz = pos[list(tri)][:, [0, 2]].mean(0)
            if np.abs(pos[p, [0, 2]] - cxz).max() < 1.5 * h:
                pairs.append((p, *tri))
                is_ee.append(0)
    for ea in bot_edges:
        for eb in top_edges:
            if np.abs(pos[list(ea)][:, [0, 2]].mean(0) - pos[list(eb)][:, [0, 2]].mean(0)).max() < 1.5 * h:
                pairs.append((*ea, *eb))
                is_ee.append(1)
    mesh = GpuTetMesh(pos, tets, c, cuda, ground=ground, ground_y=ground_y)
    return pos, tets, c, ground, ground_y, np.array(pairs, np.int32), np.array(is_ee, np.uint8), n, mesh


def test_line_search_cut_by_contact_pairs(cuda):
    """The upper cube moved down by twice its lift: the pairs between its
    bottom face and the lower cube's top face cut the step (the oracle's
    bound over the same pairs), the accepted state leaves every pair apart,
    and the line search's energy includes the pairs' barrier."""
    import torch

    from libuipc_b200.gpu_scene import GpuContacts
    from libuipc_b200.newton import line_search
    from oracle import elements as OE

    pos, tets, c, ground, ground_y, pairs, is_ee, n, mesh = _two_cubes(cuda)
    dhat, dt = c["dhat"], c["dt"]
    eps = np.full(len(pairs), 1e-12)
    C = GpuContacts(pairs, is_ee, eps, dhat, c["kappa"], dt, cuda)
    try:
        assert len(pairs) > 100 and is_ee.sum() > 20
        d = np.zeros_like(pos)
        d[n:, 1] = -2.0 * 2e-3
        x = to_dev(pos.ravel().copy(), cuda)
        xt = to_dev((pos + d).ravel().copy(), cuda)
        r = line_search(mesh, x, to_dev(d.ravel(), cuda), xt, dt, contacts=C)
        t_ref = OE.pairs_toi(pos, d, pairs, is_ee, 1.0, dhat)
        assert t_ref < 0.6 and abs(r.toi_alpha - t_ref) <= 1e-9 * t_ref
        assert r.alpha <= r.toi_alpha and not r.converged
        xa = x.cpu().numpy().reshape(-1, 3)
        # every pair still apart, and the energy the search reports is the
        # tet energy plus the pairs' barrier at the accepted state
        for p, ee in zip(pairs, is_ee):
            assert OE._pair_d2(xa[p], ee) > 0.0
        e_pairs = sum(OE.contact_energy(xa[p], ee, ep, dhat, c["kappa"] * dt * dt)
                      for p, ee, ep in zip(pairs, is_ee, eps))
        e_mesh = mesh.energy(x, xt)
        assert abs(r.energy - (e_mesh + e_pairs)) <= 1e-10 * abs(r.energy)
        assert np.isfinite(r.energy)
    finally:
        C.close()
        mesh.close()


def test_trajectory_candidates_against_brute_force(cuda):
    """The device's candidate detection (hashed uniform grid) on the whole
    surface of two stacked cubes, the upper one moving down by twice its lift
    and a little sideways: exactly the oracle's brute-force set of
    point-triangle and edge-edge pairs within dhat over the swept step (no
    pair twice, the same order on a second call); the time of impact over
    them equal to the oracle's narrow phase over the brute-force set; the
    line search with the filter cut there."""
    from libuipc_b200.gpu_scene import GpuTrajectory, tet_surface
    from libuipc_b200.newton import line_search
    from oracle import elements as OE

    pos, tets, c, ground, ground_y, _, _, n, mesh = _two_cubes(cuda)
    tris, edges, verts = tet_surface(tets)
    rng = np.random.default_rng(5)
    d = np.zeros_like(pos)
    d[n:, 1] = -2.0 * 2e-3
    d[n:, [0, 2]] = 1e-3 * rng.standard_normal(2)
    dist = c["dhat"]
    cell = float(np.linalg.norm(pos[edges[:, 0]] - pos[edges[:, 1]], axis=1).mean())
    T = GpuTrajectory(len(pos), verts, edges, tris, dist, cell, cuda)
    try:
        x, dd = to_dev(pos.ravel().copy(), cuda), to_dev(d.ravel(), cuda)
        for alpha in (1.0, 0.5):
            P, E = T.detect(x, dd, alpha)
            ref_pt, ref_ee = OE.candidate_pairs(pos, d, alpha, verts, edges, tris, dist)
            got_pt = [tuple(int(v) for v in p) for p, e in zip(P, E) if not e]
            got_ee = [tuple(int(v) for v in p) for p, e in zip(P, E) if e]
            assert len(set(got_pt)) == len(got_pt) and len(set(got_ee)) == len(got_ee)
            assert set(got_pt) == ref_pt and set(got_ee) == ref_ee
            assert len(ref_pt) > 50 and len(ref_ee) > 50
            assert (E[:len(got_pt)] == 0).all()  # point-triangle first
            P2, E2 = T.detect(x, dd, alpha)
            assert np.array_equal(P, P2) and np.array_equal(E, E2)
        ref = sorted(ref_pt) + sorted(ref_ee)  # alpha = 0.5 from the loop above
        t_ref = OE.pairs_toi(pos, d, ref, [0] * len(ref_pt) + [1] * len(ref_ee), 0.5, dist)
        t_dev = T.toi(x, dd, alpha=0.5)
        assert t_ref < 1.0 and abs(t_dev - t_ref) <= 1e-9 * t_ref
        xt = to_dev((pos + d).ravel().copy(), cuda)
        r = line_search(mesh, x, dd, xt, c["dt"], trajectory=T)
        assert r.alpha <= r.toi_alpha < 1.0
        xa = x.cpu().numpy().reshape(-1, 3)
        for p in ref_pt:
            assert OE._pair_d2(xa[list(p)], False) > 0.0
        for p in ref_ee:
            assert OE._pair_d2(xa[list(p)], True) > 0.0
    finally:
        T.close()
        mesh.close()
