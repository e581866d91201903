"""The device-side run of the twisted bar (GpuBarSequence + the GPU generator)
feeding the learned warm start: its systems match the host sequence's, and
after training on the run the history and learned starts need fewer PCG
iterations than the zero start."""
import numpy as np
import pytest

from conftest import to_dev

pytestmark = pytest.mark.gpu


def test_gpu_sequence_matches_host_sequence(solver, cuda):
    from libuipc_b200.sequence import GpuBarSequence, SceneSequence

    cfg = dict(cells_x=16, cells_y=3, cells_z=3, E=1e6, nu=0.49)
    host = SceneSequence(scene=2, twist_per_step=2.0, **cfg)
    dev = GpuBarSequence(cuda, twist_per_step=2.0, **cfg)
    try:
        for _ in range(2):
            host.begin_step()
            dev.begin_step()
            s = host.system()
            rows, cols, vals, b = dev.system()
            solver.assemble(s.n_verts, to_dev(s.rows, cuda), to_dev(s.cols, cuda), to_dev(s.vals, cuda))
            _, c1, v1 = solver.upper_bsr()
            solver.assemble(s.n_verts, rows, cols, vals)
            _, c2, v2 = solver.upper_bsr()
            assert np.array_equal(c1, c2) and np.abs(v1 - v2).max() <= 1e-11 * np.abs(v1).max()
            assert np.abs(b.cpu().numpy() - s.b).max() <= 1e-11 * np.abs(s.b).max()
            # the same update on both sides (no solve needed to compare the stepping)
            dx = 1e-4 * np.sin(np.arange(3 * s.n_verts))
            host.apply(dx)
            dev.apply(to_dev(dx, cuda))
            host.end_step()
            dev.end_step()
    finally:
        dev.close()


def test_learned_run_on_the_gpu(cuda):
    from libuipc_b200.learned import run_gpu_bar

    r = run_gpu_bar(cuda, cells=(24, 4, 4), train_steps=8, eval_steps=3, newton_iters=2, epochs=3)
    it = r["mean_pcg_iterations"]
    assert r["training_systems"] == 16 and r["eval_systems"] == 6
    assert it["history"] < it["zero"] and it["learned"] < it["zero"]


def test_stepped_full_scale_run_small(cuda):
    """The stepped cube-grid + cloth + bodies run of the bench on a small
    instance (2 x 2 cubes of 6^3 cells, 16^2 cloth, 2 x 2 bodies, 3 systems):
    every solve meets rel-res 1e-4, the systems follow the state (contact
    counts change), and the history start needs fewer PCG iterations than
    the plain solve from zero on the later systems."""
    import bench

    out = bench.full_scale_run(cuda, n_systems=3, scene_kw=dict(cells_x=6, cells_y=6, cells_z=6, n_cubes=2,
                                                                 cloth_n=16, bodies_x=2, bodies_z=2, dt=0.005,
                                                                 seed=0))
    assert len(out["systems"]) == 3 and out["timed_systems"] == 2
    for r in out["systems"]:
        for m in ("plain", "mixed+history"):
            assert r[m]["rel_res"] <= 1e-4
    for r in out["systems"][1:]:
        assert r["mixed+history"]["pcg_iterations"] < r["plain"]["pcg_iterations"]
