"""The cloth / affine-body element routines of the generators
(csrc/scene/elements.h, through libb200scene.so's b2g_element_* hooks)
against the oracle's numpy restatement of libuipc's formulas
(oracle/elements.py): energies equal, gradients equal to central differences
of the restated energies, the Baraff-Witkin Hessian equal to the reference's
closed form mapped through dF/dx, the hinge's Gauss-Newton Hessian equal to
the outer product of the finite-difference angle gradient, and the
orthogonality Hessian equal to the PSD part of the finite-difference Hessian.
Random states: stretched, compressed and sheared triangles, bent hinges,
near-rotation and general affine matrices."""
import ctypes as C

import numpy as np
import pytest

from libuipc_b200._native import load_scene_lib
from oracle import elements as OE


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _lib_bw(x, rest, stretch, shear, rate, w):
    lib = load_scene_lib()
    G, H = np.zeros(9), np.zeros(81)
    E = lib.b2g_element_bw(_ptr(np.ascontiguousarray(x)), _ptr(np.ascontiguousarray(rest)), stretch, shear, rate,
                           w, _ptr(G), _ptr(H))
    return E, G, H.reshape(9, 9)


def _lib_dsb(x, rest, kappa, w):
    lib = load_scene_lib()
    G, H = np.zeros(12), np.zeros(144)
    E = lib.b2g_element_dsb(_ptr(np.ascontiguousarray(x)), _ptr(np.ascontiguousarray(rest)), kappa, w, _ptr(G),
                            _ptr(H))
    return E, G, H.reshape(12, 12)


def _lib_ortho(q, kappa, w):
    lib = load_scene_lib()
    G, H = np.zeros(9), np.zeros(81)
    E = lib.b2g_element_ortho(_ptr(np.ascontiguousarray(q)), kappa, w, _ptr(G), _ptr(H))
    return E, G, H.reshape(9, 9)


def _close(a, b, rtol):
    return np.abs(a - b).max() <= rtol * max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("stretch_factor", [0.8, 1.0, 1.3])
def test_baraff_witkin_triangle(seed, stretch_factor):
    rng = np.random.default_rng(seed)
    rest = rng.standard_normal((3, 3)) * 0.01
    # current: rest rotated, stretched along a random in-plane direction, sheared, moved
    Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    x = rest @ Q.T
    d = rng.standard_normal(3)
    x = x + (stretch_factor - 1.0) * np.outer(x @ d / (d @ d), d) + 0.001 * rng.standard_normal((3, 3))
    stretch, shear, rate, w = 1e3, 1e2, 100.0, 3.7e-5
    E, G, H = _lib_bw(x, rest, stretch, shear, rate, w)
    Eo, Go, Ho = OE.bw_element(x, rest, stretch, shear, rate, w)
    assert abs(E - Eo) <= 1e-12 * max(abs(Eo), 1e-300) + 1e-300
    assert _close(G, Go, 1e-6)
    assert _close(H, Ho, 1e-10)
    assert np.abs(H - H.T).max() <= 1e-12 * np.abs(H).max()
    assert np.linalg.eigvalsh(H).min() >= -1e-9 * np.abs(H).max()


@pytest.mark.parametrize("seed", range(6))
def test_shell_bending_hinge(seed):
    rng = np.random.default_rng(100 + seed)
    rest = np.array([[0.0, 0.0, 1.0], [0.0, -1.0, 0.0], [0.0, 1.0, 0.0], [1.0, 0.0, 0.0]]) * 0.01
    rest = rest + 0.002 * rng.standard_normal((4, 3))
    x = rest + 0.003 * rng.standard_normal((4, 3))
    kappa, w = 1e-2, 1e-4
    E, G, H = _lib_dsb(x, rest, kappa, w)
    Eo, Go, Ho = OE.dsb_element(x, rest, kappa, w)
    assert abs(E - Eo) <= 1e-12 * max(abs(Eo), 1e-30)
    assert _close(G, Go, 1e-5)
    assert _close(H, Ho, 1e-5)
    # at the rest state: zero energy and gradient
    E0, G0, _ = _lib_dsb(rest, rest, kappa, w)
    assert E0 == 0.0 and np.abs(G0).max() == 0.0


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("kind", ["rotation", "near", "general"])
def test_orthogonality_potential(seed, kind):
    rng = np.random.default_rng(200 + seed)
    R, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    A = {"rotation": R, "near": R + 0.05 * rng.standard_normal((3, 3)),
         "general": rng.standard_normal((3, 3))}[kind]
    q = np.concatenate([rng.standard_normal(3), A.T.reshape(-1)])  # q[3+3k .. ] = column k
    kappa, w = 1e8, 2.16e-4 * 1e-4
    E, G, H = _lib_ortho(q, kappa, w)
    Eo, Go, Ho = OE.ortho_element(q, kappa, w)
    assert abs(E - Eo) <= 1e-10 * max(abs(Eo), 1e-300) + (1e-300 if kind != "rotation" else kappa * 1e-24)
    assert np.abs(G - Go).max() <= 1e-6 * np.abs(Go).max() + 1e-10 * w * kappa  # FD noise floor
    assert _close(H, Ho, 1e-5)
    assert np.linalg.eigvalsh(H).min() >= -1e-9 * np.abs(H).max()


TYPE_NAMES = {0: "PP", 1: "PE", 2: "PT", 3: "EE"}


def _lib_contact(X, is_ee, eps, dhat, k):
    lib = load_scene_lib()
    G, H = np.zeros(12), np.zeros(144)
    t = lib.b2g_element_contact(_ptr(np.ascontiguousarray(X, dtype=np.float64)), int(is_ee), eps, dhat, k, _ptr(G),
                                _ptr(H))
    return t, G, H.reshape(12, 12)


def _contact_case(kind, rng, dhat):
    """A pair of the given closest-feature type at distance 0.2-0.8 dhat."""
    d = rng.uniform(0.2, 0.8) * dhat
    R, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    h = 0.01
    if kind in ("PT", "PE", "PP"):
        t = np.array([[0, 0, 0], [h, 0, 0], [0.3 * h, h, 0]]) + 0.1 * h * rng.uniform(-1, 1, (3, 3)) * [1, 1, 0]
        if kind == "PT":
            p = t.mean(0) + [0, 0, d]
        elif kind == "PE":  # beyond the middle of edge t0t1, off the plane
            p = 0.5 * (t[0] + t[1]) + np.array([0, -d * 0.6, d * 0.8])
        else:  # beyond corner t0
            p = t[0] + np.array([-d * 0.5, -d * 0.6, d * 0.62])
        X = np.vstack([p, t])
        return (X @ R.T) + rng.standard_normal(3), 0
    # edge-edge: crossing (EE), or nearly parallel (mollified)
    a0, a1 = np.array([-h, 0, 0]), np.array([h, 0, 0])
    if kind == "EE":
        ang = rng.uniform(0.5, 1.5)
    else:
        ang = 1e-3
    b0 = np.array([-h * np.cos(ang), -h * np.sin(ang), d]) + [0.1 * h, 0, 0]
    b1 = np.array([h * np.cos(ang), h * np.sin(ang), d]) + [0.1 * h, 0, 0]
    X = np.vstack([a0, a1, b0, b1])
    return (X @ R.T) + rng.standard_normal(3), 1


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("kind", ["PT", "PE", "PP", "EE", "EE-parallel"])
def test_contact_pair(seed, kind):
    rng = np.random.default_rng(300 + seed)
    dhat, k = 1e-3, 1e9 * 1e-4
    X, is_ee = _contact_case(kind, rng, dhat)
    # mollifier threshold from the rest edges (here: the current ones)
    ea, eb = X[1] - X[0], X[3] - X[2]
    eps = 1e-3 * (ea @ ea) * (eb @ eb)
    t, G, H = _lib_contact(X, is_ee, eps, dhat, k)
    to, Go, Ho = OE.contact_element(X, is_ee, eps, dhat, k)
    want = {"EE-parallel": ("PE", "PP", "EE")}.get(kind, (kind,))
    assert TYPE_NAMES[t] == to and to in want
    assert np.abs(G - Go).max() <= 1e-5 * np.abs(Go).max()
    assert np.abs(H - Ho).max() <= 1e-4 * np.abs(Ho).max()
    assert np.abs(H - H.T).max() <= 1e-12 * np.abs(H).max()
    assert np.linalg.eigvalsh(H).min() >= -1e-9 * np.abs(H).max()
    if kind == "EE-parallel":  # the mollifier is active
        c = np.cross(ea, eb)
        assert c @ c < eps


def test_contact_beyond_dhat_is_zero():
    X = np.array([[0, 0, 2e-3], [0, 0, 0], [0.01, 0, 0], [0, 0.01, 0]], np.float64)
    t, G, H = _lib_contact(X, 0, 0.0, 1e-3, 1e5)
    assert t == -1 and not G.any() and not H.any()


def _lib_energy(X, is_ee, eps, dhat, k):
    return load_scene_lib().b2g_contact_energy(_ptr(np.ascontiguousarray(X, dtype=np.float64)), int(is_ee), eps,
                                               dhat, k)


def _lib_accd(X, dX, is_ee, eta=0.1, xi=0.0, max_iter=1000, toi_max=1.1):
    t = C.c_double()
    hit = load_scene_lib().b2g_accd(_ptr(np.ascontiguousarray(X, dtype=np.float64)),
                                    _ptr(np.ascontiguousarray(dX, dtype=np.float64)), int(is_ee), eta, xi, max_iter,
                                    toi_max, C.byref(t))
    return bool(hit), t.value


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("kind", ["PT", "PE", "PP", "EE", "EE-parallel"])
def test_contact_energy(seed, kind):
    """The barrier energy (times the mollifier for near-parallel edges) equals
    the oracle's, and its central difference is the element's gradient."""
    rng = np.random.default_rng(500 + seed)
    dhat, k = 1e-3, 1e9 * 1e-4
    X, is_ee = _contact_case(kind, rng, dhat)
    ea, eb = X[1] - X[0], X[3] - X[2]
    eps = 1e-3 * (ea @ ea) * (eb @ eb)
    e = _lib_energy(X, is_ee, eps, dhat, k)
    eo = OE.contact_energy(X, is_ee, eps, dhat, k)
    assert eo > 0 and abs(e - eo) <= 1e-12 * eo
    _, G, _ = _lib_contact(X, is_ee, eps, dhat, k)
    h = 1e-4 * dhat
    fd = np.zeros(12)
    for i in range(12):
        Xp, Xm = X.copy().reshape(-1), X.copy().reshape(-1)
        Xp[i] += h
        Xm[i] -= h
        fd[i] = (_lib_energy(Xp.reshape(4, 3), is_ee, eps, dhat, k) - _lib_energy(Xm.reshape(4, 3), is_ee, eps, dhat,
                                                                                 k)) / (2 * h)
    assert np.abs(fd - G).max() <= 1e-4 * np.abs(G).max()


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("kind", ["PT", "PE", "PP", "EE", "EE-parallel"])
def test_additive_ccd(seed, kind):
    """Additive CCD of a pair under random relative motion of a few times its
    distance: hit and time of impact equal to the oracle's (to rounding), the
    pair still apart at the time of impact, and no hit for pure translation."""
    rng = np.random.default_rng(700 + seed)
    dhat = 1e-3
    X, is_ee = _contact_case(kind, rng, dhat)
    hits = 0
    for trial in range(8):
        dX = rng.standard_normal((4, 3)) * dhat * rng.uniform(0.5, 4.0)
        hit, t = _lib_accd(X, dX, is_ee)
        ho, to = OE.accd_toi(X, dX, is_ee)
        assert hit == ho and abs(t - to) <= 1e-13 * to
        if hit:
            hits += 1
            assert 0.0 <= t <= 1.1
            assert OE._pair_d2(X + t * dX, is_ee) > 0.0
    assert _lib_accd(X, np.tile(rng.standard_normal(3), (4, 1)), is_ee) == (False, 1.1)


def test_additive_ccd_straight_approach():
    """A point 1 mm above a triangle moving 2 mm down along the normal: the
    first advance covers (1 - eta) of the distance, the next one ends below
    eta of it, so the time of impact is (1 - eta) / 2."""
    X = np.array([[0.2e-2, 1e-3, 0.2e-2], [0.0, 0.0, 0.0], [1e-2, 0.0, 0.0], [0.0, 0.0, 1e-2]])
    dX = np.zeros((4, 3))
    dX[0, 1] = -2e-3
    hit, t = _lib_accd(X, dX, 0)
    assert hit and abs(t - 0.45) <= 1e-15
    # moving away: no hit
    assert _lib_accd(X, -dX, 0) == (False, 1.1)
