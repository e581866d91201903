"""The line search after the solve (libuipc_b200/newton.py, b2gen_energy,
b2gen_ground_toi) on a cube dropped onto the ground: the device energy
against the oracle's numpy restatement, the ground's time of impact against a
direct computation, and a run of Newton steps (solve, line search) in which
every accepted step lowers the energy (or the iteration had converged), no
vertex crosses the ground and the fall is slowed by it."""
import numpy as np
import pytest

from conftest import to_dev

pytestmark = pytest.mark.gpu


def _cube(cuda, cells=6):
    from libuipc_b200 import scene
    from libuipc_b200.gpu_scene import GpuTetMesh

    s = scene.cube_on_ground(cells, seed=2)
    c = s.config
    vx = vy = cells + 1
    v = np.arange(s.n_verts)
    bottom = v[(v // vx) % vy == 0].astype(np.int32)
    ground_y = s.positions[bottom, 1].min() - c["ground_offset"]
    mesh = GpuTetMesh(s.positions, s.tets, c, cuda, ground=bottom, ground_y=ground_y)
    return s, c, bottom, ground_y, mesh


def test_energy_and_time_of_impact(cuda):
    import torch

    from oracle import elements as OE

    s, c, bottom, ground_y, mesh = _cube(cuda)
    try:
        E, nu = c["E"], c["nu"]
        mu, lam = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
        rng = np.random.default_rng(0)
        x = s.positions + 1e-4 * rng.standard_normal(s.positions.shape)
        x[bottom, 1] = np.maximum(x[bottom, 1], ground_y + 2e-4)
        xt = s.positions.copy()
        xt[:, 1] -= c["dt"] ** 2 * c["gravity"]
        e_dev = mesh.energy(to_dev(x.ravel(), cuda), to_dev(xt.ravel(), cuda))
        e_ref = OE.tet_energy(s.positions, s.tets, x, xt, mu, lam, c["rho"], c["dt"], ground=bottom,
                              ground_y=ground_y, dhat=c["dhat"], kappa=c["kappa"])
        assert abs(e_dev - e_ref) <= 1e-10 * abs(e_ref)
        # a vertex below the plane: infinite energy
        xb = x.copy()
        xb[bottom[0], 1] = ground_y - 1e-6
        assert mesh.energy(to_dev(xb.ravel(), cuda), to_dev(xt.ravel(), cuda)) == float("inf")
        # time of impact: the bottom moving down by twice its height above the ground
        d = np.zeros_like(x)
        d[:, 1] = -2.0 * (x[:, 1] - ground_y)
        toi = mesh.ground_toi(to_dev(x.ravel(), cuda), to_dev(d.ravel(), cuda))
        assert abs(toi - 0.9 * 0.5) <= 1e-12
        d[:, 1] = 1e-3  # moving up: no impact
        assert mesh.ground_toi(to_dev(x.ravel(), cuda), to_dev(d.ravel(), cuda)) == 1.0
    finally:
        mesh.close()


def test_newton_steps_with_line_search(solver, cuda):
    import torch

    from libuipc_b200 import _abi
    from libuipc_b200.linear_system import partition_maps, partition_rcb
    from libuipc_b200.newton import line_search

    s, c, bottom, ground_y, mesh = _cube(cuda)
    try:
        dt, g = c["dt"], c["gravity"]
        p2r, r2p = partition_maps(partition_rcb(s.positions))
        solver.mas_init(0, s.n_verts, s.adj_start, s.adj_list, p2r, r2p)
        x = to_dev(s.positions.ravel().copy(), cuda)
        v = torch.zeros_like(x)
        v[1::3] = -0.5  # dropped onto the ground at 0.5 m/s
        min_gap = float("inf")
        for step in range(12):
            x_prev = x.clone()
            xt = x + dt * v
            xt[1::3] -= dt * dt * g
            for _ in range(4):
                rows, cols, vals, b = mesh.system(x, xt)
                solver.assemble(s.n_verts, rows, cols, vals)
                solver.precond_assemble(_abi.B2S_PRECOND_MAS)
                sol = torch.zeros_like(b)
                st = solver.pcg(b, sol, tol=1e-6, stop_rule=_abi.B2S_STOP_RELRES)
                assert st["converged"] == 1
                r = line_search(mesh, x, -sol, xt, dt)
                assert 0.0 < r.alpha <= 1.0
                assert r.converged or r.energy <= r.energy0
                if r.converged:
                    assert r.alpha == 1.0 and r.trials == 1
                gap = float((x[1::3][torch.as_tensor(bottom, device=cuda)] - ground_y).min())
                assert gap > 0.0
                min_gap = min(min_gap, gap)
            v = (x - x_prev) / dt
        # the cube reached the barrier's range and the ground slowed its fall
        assert min_gap < c["dhat"]
        assert float(v[1::3].abs().max()) < 0.45
    finally:
        mesh.close()
