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
