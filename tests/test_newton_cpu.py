"""The line search's host logic (libuipc_b200/newton.py) and the oracle's
continuous collision detection (oracle/elements.py), on the CPU.

* line_search with stand-in mesh / contact objects (numpy, no device): the
  step starts at min(1, ground time of impact, contact time of impact), the
  energy it tests is the mesh's plus the contacts', it halves until the
  energy does not rise and keeps the last trial, and a converged iteration
  (largest displacement below velocity_tol dt, no cut) takes its first trial.
* the additive CCD is conservative against the exact time of impact of a
  point moving on a straight line towards a fixed triangle, and of two edges
  closing on a straight line: it never passes the contact and stops within
  (1 - eta) of it, and the pair is still apart at the time it returns."""
import numpy as np
import pytest

from libuipc_b200.newton import line_search
from oracle import elements as OE


class _Vec:
    """The few tensor methods line_search uses, over a numpy array."""

    def __init__(self, a):
        self.a = np.array(a, dtype=np.float64)

    def clone(self):
        return _Vec(self.a)

    def copy_(self, o):
        self.a[:] = o.a
        return self

    def add_(self, o, alpha=1.0):
        self.a += alpha * o.a
        return self

    def abs(self):
        return _Vec(np.abs(self.a))

    def max(self):
        return float(self.a.max())

    def reshape(self, *shape):
        return self.a.reshape(*shape)


class _Mesh:
    """E(x) = 1/2 |x - target|^2; the ground cuts at `ground_toi`."""

    def __init__(self, target, ground_toi=1.0):
        self.target, self.g = np.asarray(target, dtype=np.float64), ground_toi
        self.energy_calls = 0

    def energy(self, x, x_tilde):
        self.energy_calls += 1
        return 0.5 * float(((x.a - self.target) ** 2).sum())

    def ground_toi(self, x, d):
        return self.g


class _Contacts:
    def __init__(self, toi, barrier):
        self.t, self.barrier = toi, barrier

    def energy(self, x):
        return self.barrier(x.a)

    def toi(self, x, d):
        return self.t


def test_step_starts_at_the_smallest_time_of_impact():
    x = _Vec([0.0, 0.0])
    d = _Vec([1.0, 0.0])
    mesh = _Mesh([1.0, 0.0], ground_toi=0.8)
    r = line_search(mesh, x, d, None, dt=1.0, velocity_tol=0.0, contacts=_Contacts(0.3, lambda a: 0.0))
    assert r.toi_alpha == 0.3 and r.alpha == 0.3 and r.trials == 1
    assert np.allclose(x.a, [0.3, 0.0])
    r = line_search(mesh, _Vec([0.0, 0.0]), d, None, dt=1.0, velocity_tol=0.0)  # ground only
    assert r.toi_alpha == 0.8 and r.alpha == 0.8


def test_energy_includes_the_contacts_and_halves_until_it_does_not_rise():
    # the mesh alone accepts alpha = 1; a barrier rising steeply past x0 = 0.3
    # rejects 1 and 0.5 and accepts 0.25
    def barrier(a):
        return 0.0 if a[0] <= 0.3 else 1e3 * (a[0] - 0.3)

    x = _Vec([0.0])
    mesh = _Mesh([1.0])
    r = line_search(mesh, x, _Vec([1.0]), None, dt=1.0, velocity_tol=0.0, contacts=_Contacts(1.0, barrier))
    assert r.alpha == 0.25 and r.trials == 3
    assert r.energy == pytest.approx(0.5 * 0.75 ** 2) and r.energy0 == pytest.approx(0.5)
    assert not r.converged


def test_no_decrease_keeps_the_last_trial():
    x = _Vec([0.0])
    mesh = _Mesh([-1.0])  # every step along +d raises the energy
    r = line_search(mesh, x, _Vec([1.0]), None, dt=1.0, velocity_tol=0.0, max_iter=4)
    assert r.trials == 4 and r.alpha == 0.125 and x.a[0] == 0.125


def test_converged_iteration_takes_its_first_trial():
    x = _Vec([0.0])
    mesh = _Mesh([-1.0])
    r = line_search(mesh, x, _Vec([1e-4]), None, dt=0.01, velocity_tol=0.05,
                    contacts=_Contacts(1.0, lambda a: 0.0))
    assert r.converged and r.trials == 1 and r.alpha == 1.0
    # a step cut by a time of impact is not converged
    r = line_search(mesh, _Vec([0.0]), _Vec([1e-4]), None, dt=0.01, velocity_tol=0.05,
                    contacts=_Contacts(0.5, lambda a: 0.0))
    assert not r.converged


@pytest.mark.parametrize("seed", range(20))
def test_ccd_point_triangle_is_conservative(seed):
    rng = np.random.default_rng(seed)
    t = rng.uniform(-1, 1, (3, 3)) * [1, 0.05, 1]
    n = np.cross(t[1] - t[0], t[2] - t[0])
    n /= np.linalg.norm(n)
    w = rng.dirichlet([2, 2, 2])
    inside = w @ t
    h = 10 ** rng.uniform(-4, -1)
    p = inside + h * n
    speed = rng.uniform(1.2, 5.0)  # the step covers 1.2-5x the distance to the face
    dp = -speed * h * n + 0.1 * h * rng.standard_normal(3) * [1, 0, 1]
    X = np.vstack([p, t])
    dX = np.zeros((4, 3))
    dX[0] = dp
    # exact time the point reaches the triangle's plane (still inside the face)
    t_exact = h / -(dp @ n)
    hit, toi = OE.accd_toi(X, dX, False)
    assert hit and toi <= t_exact and toi >= 0.8 * t_exact
    assert OE._pair_d2(X + toi * dX, False) > 0.0


@pytest.mark.parametrize("seed", range(20))
def test_ccd_edge_edge_is_conservative(seed):
    rng = np.random.default_rng(100 + seed)
    a0, a1 = np.array([-1.0, 0, 0]), np.array([1.0, 0, 0])
    ang = rng.uniform(0.3, np.pi - 0.3)
    h = 10 ** rng.uniform(-4, -1)
    b0 = np.array([-np.cos(ang), h, -np.sin(ang)]) * [0.8, 1, 0.8]
    b1 = np.array([np.cos(ang), h, np.sin(ang)]) * [0.8, 1, 0.8]
    b0[1] = b1[1] = h
    speed = rng.uniform(1.2, 5.0)
    X = np.vstack([a0, a1, b0, b1])
    dX = np.zeros((4, 3))
    dX[2:, 1] = -speed * h
    hit, toi = OE.accd_toi(X, dX, True)
    t_exact = 1.0 / speed  # the crossing edges meet when b reaches y = 0
    assert hit and toi <= t_exact and toi >= 0.8 * t_exact
    assert OE._pair_d2(X + toi * dX, True) > 0.0


def test_ccd_no_hit_when_the_step_stops_short():
    X = np.array([[0.1, 1e-2, 0.1], [0, 0, 0], [1, 0, 0], [0, 0, 1]], dtype=np.float64)
    dX = np.zeros((4, 3))
    dX[0, 1] = -0.5e-2  # half way down
    assert OE.accd_toi(X, dX, False) == (False, 1.1)
    assert OE.pairs_toi(X, dX, [[0, 1, 2, 3]], [False], 1.0, dhat=1e-3) == 1.0
    # far apart: the swept boxes do not meet, whatever the CCD would say
    assert not OE.ccd_broadphase(X + [0, 5, 0], dX, False, 1e-3)


def test_tet_surface_of_a_cube():
    """The boundary of an n^3-cell tet cube: 2 triangles per face cell, every
    boundary grid vertex, and every boundary edge shared by two boundary
    triangles (a closed surface: V - E + F = 2)."""
    from libuipc_b200 import scene
    from libuipc_b200.gpu_scene import tet_surface

    n = 3
    s = scene.cube_on_ground(n, seed=0)
    tris, edges, verts = tet_surface(s.tets)
    assert len(tris) == 6 * 2 * n * n
    assert len(verts) == (n + 1) ** 3 - (n - 1) ** 3
    assert len(verts) - len(edges) + len(tris) == 2
    e = np.sort(np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [0, 2]]]), axis=1)
    _, cnt = np.unique(e, axis=0, return_counts=True)
    assert (cnt == 2).all()


def test_candidate_pairs_brute_force():
    """The oracle's candidate set on a small case: a vertex over a triangle
    within dist is a pair, farther is not, a pair sharing a vertex never is,
    and crossing edges within dist are a pair in one orientation only."""
    x = np.array([[0.2, 1e-3, 0.2], [0, 0, 0], [1, 0, 0], [0, 0, 1], [0.2, 5e-3, 0.2]], dtype=np.float64)
    dx = np.zeros_like(x)
    tris = np.array([[1, 2, 3]])
    pt, ee = OE.candidate_pairs(x, dx, 1.0, [0, 4], np.zeros((0, 2), int), tris, 2e-3)
    assert pt == {(0, 1, 2, 3)}
    # moving the far vertex down brings it in
    dx[4, 1] = -4e-3
    pt, _ = OE.candidate_pairs(x, dx, 1.0, [0, 4], np.zeros((0, 2), int), tris, 2e-3)
    assert pt == {(0, 1, 2, 3), (4, 1, 2, 3)}
    # edges: (1, 2) and (0, 4) cross near x = 0.2; (1, 3) shares vertex 1 with (1, 2)
    edges = np.array([[1, 2], [1, 3], [0, 4]])
    y = x.copy()
    y[0] = [0.2, 1e-3, -0.5]
    y[4] = [0.2, 1e-3, 0.5]
    _, ee = OE.candidate_pairs(y, np.zeros_like(y), 1.0, [], edges, np.zeros((0, 3), int), 2e-3)
    assert ee == {(1, 2, 0, 4)}


def test_cfl_bound_and_its_use():
    """0.5 dhat over the largest (surface) vertex displacement, capped at 1;
    the line search applies it only when a time of impact cut the step."""
    from libuipc_b200.newton import cfl_bound

    d = np.array([[0.0, -2e-3, 0.0], [0.0, 0.0, 1e-3], [0.0, 0.0, 0.0]])
    assert cfl_bound(d, 1e-3) == pytest.approx(0.25)
    assert cfl_bound(d, 1e-3, verts=[1, 2]) == pytest.approx(0.5)
    assert cfl_bound(d, 1e-2) == 1.0 and cfl_bound(np.zeros((2, 3)), 1e-3) == 1.0
    x = _Vec(np.zeros(9))
    dv = _Vec(d.ravel())
    mesh = _Mesh(d.ravel())  # the energy falls all the way along d
    r = line_search(mesh, x, dv, None, dt=1.0, velocity_tol=0.0, contacts=_Contacts(0.8, lambda a: 0.0),
                    cfl_dhat=1e-3)
    assert r.toi_alpha == 0.8 and r.alpha == pytest.approx(0.25)
    r = line_search(mesh, _Vec(np.zeros(9)), dv, None, dt=1.0, velocity_tol=0.0,
                    contacts=_Contacts(1.0, lambda a: 0.0), cfl_dhat=1e-3)
    assert r.alpha == 1.0  # no cut by a time of impact: no CFL cap
