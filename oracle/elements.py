"""CPU oracle (test infrastructure) of the cloth / affine-body element
energies the generators produce: a numpy restatement of libuipc's formulas,
written independently of the library's C++ (csrc/scene/elements.h), used only
by tests to check it.

* Baraff-Witkin shell: strain_limiting_baraff_witkin_shell_2d.h:33-280 (rest
  frame Dm2x2 :33-66, E :96-127, dEdF :129-170, ddEddF :172-278) and the
  element assembly of strain_limiting_baraff_witkin_shell_2d.cu:75-150
  (G = dFdx^T vec(dEdF), H = dFdx^T ddEddF dFdx, weight rest area dt^2).
* Discrete-shell bending: discrete_shell_bending_function.h:33-135 (Gauss-
  Newton Hessian), discrete_shell_bending_reference.h:8-28 (rest L0, h_bar,
  theta_bar), utils/dihedral_angle.h:14-60 (angle and its gradient).
* Affine-body orthogonality potential: affine_body/constitutions/
  sym/ortho_potential.inl (E, dEdq, ddEddq over q[3..11]),
  ortho_potential.cu:37-70 (make_spd on the 9x9, weight volume dt^2).
* IPC normal contact of a point-triangle / edge-edge pair:
  utils/distance/distance_flagged.h:258-360 (point-triangle closest-feature
  flags), the squared distances of each type, the barrier
  sym/codim_ipc_contact.inl:5-110 (thickness 0), the edge-edge mollifier
  utils/distance/details/edge_edge_mollifier.inl:63-78, 498-507, and the
  default Hessian mode of ipc_simplex_normal_contact.cu:320-360 (exact
  Hessian + PSD projection for PT / EE and mollified pairs, the closed form
  (B'' + B'/(2D)) grad D grad D^T for PE / PP). The distance derivatives
  here are central differences of the closed-form distances in 50-digit
  arithmetic (mpmath).
* The line search's contact term: the pairs' barrier energy, the trajectory
  filter's far test of swept boxes (utils/distance/details/ccd.inl
  *_ccd_broadphase), a brute-force candidate enumeration, and additive CCD
  (ccd.inl point_triangle_ccd / edge_edge_ccd, the published conservative
  advancement of Li et al. 2021) with the filter's constants
  (collision_detection/filters/lbvh_simplex_trajectory_filter.cu:18-21,
  876-1010; global_trajectory_filter.cu:111-134).
"""
from __future__ import annotations

import numpy as np


# ---- Baraff-Witkin -------------------------------------------------------------
def bw_rest(x0, x1, x2):
    """Dm^-1 of the rest triangle in its own uv frame (normal rotated to +z)."""
    n = np.cross(x1 - x0, x2 - x0)
    n = n / np.linalg.norm(n)
    z = np.array([0.0, 0.0, 1.0])
    v = np.cross(n, z)
    c = float(n @ z)
    R = np.eye(3)
    if c + 1 == 0:
        R[0, 0] = R[1, 1] = -1.0
    else:
        K = np.array([[0, -v[2], v[1]], [v[2], 0, -v[0]], [-v[1], v[0], 0]])
        R = R + K + K @ K / (1 + c)
    uv = [(R @ p)[:2] for p in (x0, x1, x2)]
    Dm = np.column_stack([uv[1] - uv[0], uv[2] - uv[0]])
    return np.linalg.inv(Dm)


def bw_F(x, IB):
    Ds = np.column_stack([x[1] - x[0], x[2] - x[0]])
    return Ds @ IB


def bw_energy(F, stretch, shear, rate):
    a, b = np.array([1.0, 0.0]), np.array([0.0, 1.0])
    I6 = a @ F.T @ F @ b
    ru, rv = np.linalg.norm(F @ a), np.linalg.norm(F @ b)
    cu, cv = (0.0 if ru <= 1 else 1.0), (0.0 if rv <= 1 else 1.0)
    st = (ru - 1) ** 2 + cu * rate * (ru - 1) ** 3 + (rv - 1) ** 2 + cv * rate * (rv - 1) ** 3
    return stretch * st + shear * I6 * I6


def bw_ddEddF(F, stretch, shear, rate):
    a, b = np.array([1.0, 0.0]), np.array([0.0, 1.0])
    Hs = np.zeros((6, 6))
    I5u = max(float((F @ a) @ (F @ a)), 1e-12)
    I5v = max(float((F @ b) @ (F @ b)), 1e-12)
    su, sv = np.sqrt(I5u), np.sqrt(I5v)
    if su > 1:
        Hs[0:3, 0:3] += np.eye(3) * 2 * ((su - 1) * (3 * su * rate - 3 * rate + 2) / (2 * su))
    if sv > 1:
        Hs[3:6, 3:6] += np.eye(3) * 2 * ((sv - 1) * (3 * sv * rate - 3 * rate + 2) / (2 * sv))
    fu = F[:, 0] / np.linalg.norm(F[:, 0])
    fv = F[:, 1] / np.linalg.norm(F[:, 1])
    uc = (3 * I5u * rate - 3 * rate + 2) / np.sqrt(I5u) if su > 1 else 2.0
    vc = (3 * I5v * rate - 3 * rate + 2) / np.sqrt(I5v) if sv > 1 else 2.0
    Hs[0:3, 0:3] += uc * np.outer(fu, fu)
    Hs[3:6, 3:6] += vc * np.outer(fv, fv)
    S = np.zeros((6, 6))
    S[3, 0] = S[4, 1] = S[5, 2] = S[0, 3] = S[1, 4] = S[2, 5] = 1.0
    I6 = a @ F.T @ F @ b
    sg = 1.0 if I6 >= 0 else -1.0
    g = F @ (np.outer(a, b) + np.outer(b, a))
    vg = np.concatenate([g[:, 0], g[:, 1]])
    I2 = float((F * F).sum())
    lam0 = 0.5 * (I2 + np.sqrt(I2 * I2 + 12 * I6 * I6))
    q0 = I6 * S @ vg + lam0 * vg
    q0 = q0 / np.linalg.norm(q0)
    T = 0.5 * (np.eye(6) + sg * S)
    Tq = T @ q0
    Hsh = 2 * (abs(I6) * (T - np.outer(Tq, Tq) / (Tq @ Tq)) + lam0 * np.outer(q0, q0))
    return stretch * Hs + shear * Hsh


def bw_dFdx(IB):
    d0, d1, d2, d3 = IB[0, 0], IB[1, 0], IB[0, 1], IB[1, 1]
    D = np.zeros((6, 9))
    for i in range(3):
        D[i, i] = -(d0 + d1)
        D[i + 3, i] = -(d2 + d3)
        D[i, i + 3] = d0
        D[i + 3, i + 3] = d2
        D[i, i + 6] = d1
        D[i + 3, i + 6] = d3
    return D


def bw_element(x, rest, stretch, shear, rate, w):
    """(E, G[9], H[9x9]) of one triangle: E unscaled, G and H scaled by w.
    G by central differences of E (an independent check of the closed forms)."""
    IB = bw_rest(*rest)
    D = bw_dFdx(IB)
    H = w * D.T @ bw_ddEddF(bw_F(x, IB), stretch, shear, rate) @ D
    E = bw_energy(bw_F(x, IB), stretch, shear, rate)
    def e(k, d):
        xx = x.copy()
        xx[k // 3, k % 3] += d
        return bw_energy(bw_F(xx, IB), stretch, shear, rate)

    h = 1e-6 * np.abs(x).max()
    # fourth-order central differences
    G = np.array([w * (8 * (e(k, h) - e(k, -h)) - (e(k, 2 * h) - e(k, -2 * h))) / (12 * h) for k in range(9)])
    return E, G, H


# ---- discrete-shell bending ---------------------------------------------------
def dihedral(x0, x1, x2, x3):
    n1 = np.cross(x1 - x0, x2 - x0)
    n2 = np.cross(x2 - x3, x1 - x3)
    c = np.clip(n1 @ n2 / np.sqrt((n1 @ n1) * (n2 @ n2)), -1.0, 1.0)
    th = np.arccos(c)
    return -th if np.cross(n2, n1) @ (x1 - x2) < 0 else th


def dsb_rest(x0, x1, x2, x3):
    L0 = np.linalg.norm(x2 - x1)
    A = (np.linalg.norm(np.cross(x1 - x0, x2 - x0)) + np.linalg.norm(np.cross(x2 - x3, x1 - x3))) / 2
    return L0, A / 3 / L0, dihedral(x0, x1, x2, x3)


def dsb_element(x, rest, kappa, w):
    """(E, G[12], H_GN[12x12]): the angle gradient by central differences."""
    L0, hb, thb = dsb_rest(*rest)
    th = dihedral(*x)
    E = L0 * kappa * (th - thb) ** 2 / hb
    g = np.zeros(12)
    h = 1e-7
    for k in range(12):
        xp, xm = x.copy(), x.copy()
        xp[k // 3, k % 3] += h
        xm[k // 3, k % 3] -= h
        g[k] = (dihedral(*xp) - dihedral(*xm)) / (2 * h)
    G = w * 2 * L0 * kappa * (th - thb) / hb * g
    H = w * 2 * L0 * kappa / hb * np.outer(g, g)
    return E, G, H


# ---- affine-body orthogonality ------------------------------------------------
def ortho_energy(q, kappa):
    a = [q[3:6], q[6:9], q[9:12]]
    return kappa * sum((a[i] @ a[j] - (i == j)) ** 2 for i in range(3) for j in range(3))


def ortho_element(q, kappa, w):
    """(E, G[9], H[9x9]): G and the Hessian by central differences of E, the
    Hessian then projected to PSD by numpy's eigh."""
    E = ortho_energy(q, kappa)
    h = 1e-6

    def grad(qq):
        g = np.zeros(9)
        for k in range(9):
            qp, qm = qq.copy(), qq.copy()
            qp[3 + k] += h
            qm[3 + k] -= h
            g[k] = (ortho_energy(qp, kappa) - ortho_energy(qm, kappa)) / (2 * h)
        return g

    G = w * grad(q)
    # second derivatives of E by central differences of E (E is a quartic
    # polynomial: the differences are exact up to rounding), then the PSD part
    H = np.zeros((9, 9))
    hh = 1e-4
    for k in range(9):
        for l in range(9):
            def e(dk, dl):
                qq = q.copy()
                qq[3 + k] += dk
                qq[3 + l] += dl
                return ortho_energy(qq, kappa)
            H[k, l] = (e(hh, hh) - e(hh, -hh) - e(-hh, hh) + e(-hh, -hh)) / (4 * hh * hh)
    wv, V = np.linalg.eigh(0.5 * (H + H.T))
    H = (V * np.maximum(wv, 0)) @ V.T
    return E, G, w * H


# ---- IPC normal contact ---------------------------------------------------------
# the squared distances written for any number type (float or mpmath mpf), so
# that their derivatives can be taken by central differences in 50-digit
# arithmetic (near-parallel edges make the line-line distance ill-conditioned
# in double precision)
def _sub(a, b):
    return [a[0] - b[0], a[1] - b[1], a[2] - b[2]]


def _crs(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def _dt(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _d2_pp(a, b):
    d = _sub(a, b)
    return _dt(d, d)


def _d2_pe(p, e0, e1):
    e = _sub(e1, e0)
    c = _crs(_sub(p, e0), e)
    return _dt(c, c) / _dt(e, e)


def _d2_plane(q, a0, u, v):
    n = _crs(u, v)
    return _dt(_sub(q, a0), n) ** 2 / _dt(n, n)


def pt_type(X):
    """(type, local vertices) of a point-triangle pair X[4, 3] = (p, t0, t1, t2)."""
    p, t = X[0], X[1:]
    n = np.cross(t[1] - t[0], t[2] - t[0])
    s, out = [], []
    for k in range(3):
        a, b = t[k], t[(k + 1) % 3]
        e = b - a
        o = np.cross(e, n)
        w = p - a
        s.append(w @ e / (e @ e))
        out.append(w @ o / (o @ o) >= 0)
    for k in range(3):
        if 0 < s[k] < 1 and out[k]:
            return "PE", [0, 1 + k, 1 + (k + 1) % 3]
    for k in range(3):
        if s[k] <= 0 and s[(k + 2) % 3] >= 1:
            return "PP", [0, 1 + k]
    return "PT", [0, 1, 2, 3]


def ee_type(X):
    a0, a1, b0, b1 = X
    u, w, z = a1 - a0, b1 - b0, a0 - b0
    a, b, c, d, e = u @ u, u @ w, w @ w, u @ z, w @ z
    den = a * c - b * b
    ux = np.cross(u, w)
    if not (ux @ ux <= 1e-12 * a * c):
        sN, tN = b * e - c * d, a * e - b * d
        if 0 < sN < den and 0 < tN < den:
            return "EE", [0, 1, 2, 3]
    best, bv = np.inf, None
    for pi, s0, s1 in ((0, 2, 3), (1, 2, 3), (2, 0, 1), (3, 0, 1)):
        P, S0, S1 = X[pi], X[s0], X[s1]
        sv = S1 - S0
        t = (P - S0) @ sv / (sv @ sv)
        if t <= 0 or t >= 1:
            Q = S0 if t <= 0 else S1
            dist, vv = float((P - Q) @ (P - Q)), [pi, s0 if t <= 0 else s1]
        else:
            q = P - S0 - t * sv
            dist, vv = float(q @ q), [pi, s0, s1]
        if dist < best:
            best, bv = dist, vv
    return ("PP" if len(bv) == 2 else "PE"), bv


def _dist(X, kind, v):
    if kind == "PP":
        return _d2_pp(X[v[0]], X[v[1]])
    if kind == "PE":
        return _d2_pe(X[v[0]], X[v[1]], X[v[2]])
    if kind == "PT":
        return _d2_plane(X[0], X[1], _sub(X[2], X[1]), _sub(X[3], X[1]))
    return _d2_plane(X[2], X[0], _sub(X[1], X[0]), _sub(X[3], X[2]))


def _fd_grad_hess(f, X):
    """Gradient and Hessian of f(X[4][3]) by central differences in 50-digit
    arithmetic."""
    import mpmath as mp

    with mp.workdps(50):
        x0 = [mp.mpf(float(c)) for c in np.asarray(X, dtype=np.float64).reshape(-1)]
        h = mp.mpf(1e-15) * max(abs(c) for c in x0)

        def F(dx):
            x = [x0[i] + dx.get(i, 0) for i in range(12)]
            return f([x[0:3], x[3:6], x[6:9], x[9:12]])
        g = np.zeros(12)
        H = np.zeros((12, 12))
        for i in range(12):
            g[i] = float((F({i: h}) - F({i: -h})) / (2 * h))
            for j in range(i, 12):
                def e(di, dj):
                    d = {i: di}
                    d[j] = d.get(j, 0) + dj
                    return F(d)
                H[i, j] = H[j, i] = float((e(h, h) - e(h, -h) - e(-h, h) + e(-h, -h)) / (4 * h * h))
    return g, H


def barrier(D, Dh, k):
    t, l = D - Dh, np.log(D / Dh)
    return -k * t * t * l, -k * (2 * t * l + t * t / D), -k * (2 * l + 4 * t / D - t * t / D ** 2)


def contact_element(X, is_ee, eps, dhat, k):
    """(type, G[12], H[12x12]) of one pair X[4, 3]."""
    X = np.asarray(X, dtype=np.float64).reshape(4, 3)
    kind, v = ee_type(X) if is_ee else pt_type(X)
    D = float(_dist([list(r) for r in X], kind, v))
    Dh = dhat * dhat
    if not (0 < D < Dh):
        return None, np.zeros(12), np.zeros((12, 12))
    gD, HD = _fd_grad_hess(lambda x: _dist(x, kind, v), X)
    B0, B1, B2 = barrier(D, Dh, k)
    moll = False
    if is_ee:
        c = np.cross(X[1] - X[0], X[3] - X[2])
        moll = c @ c < eps
    if moll:
        def cfun(x):
            c = _crs(_sub(x[1], x[0]), _sub(x[3], x[2]))
            return _dt(c, c)
        cv = float(cfun([list(r) for r in X]))
        gc, Hc = _fd_grad_hess(cfun, X)
        xx = cv / eps
        m0, m1, m2 = (2 - xx) * xx, 2 / eps * (1 - xx), -2 / eps ** 2
        gm, Hm = m1 * gc, m1 * Hc + m2 * np.outer(gc, gc)
        gB, HB = B1 * gD, B2 * np.outer(gD, gD) + B1 * HD
        G = m0 * gB + B0 * gm
        H = m0 * HB + np.outer(gm, gB) + np.outer(gB, gm) + B0 * Hm
    elif kind in ("PT", "EE"):
        G = B1 * gD
        H = B2 * np.outer(gD, gD) + B1 * HD
    else:
        return kind, B1 * gD, (B2 + B1 / (2 * D)) * np.outer(gD, gD)
    w, V = np.linalg.eigh(0.5 * (H + H.T))
    return kind, G, (V * np.maximum(w, 0)) @ V.T


def _pair_d2(X, is_ee):
    kind, v = ee_type(X) if is_ee else pt_type(X)
    return float(_dist([list(r) for r in X], kind, v))


def contact_energy(X, is_ee, eps, dhat, k):
    """Barrier energy of one pair X[4, 3] (k = kappa dt^2): B(D) of its
    closest-feature squared distance, times the edge-edge mollifier
    (2 - c/eps) c/eps, c = |ea x eb|^2, below eps; 0 at or beyond dhat."""
    X = np.asarray(X, dtype=np.float64).reshape(4, 3)
    D, Dh = _pair_d2(X, is_ee), dhat * dhat
    if not (0 < D < Dh):
        return 0.0
    B0 = barrier(D, Dh, k)[0]
    if is_ee:
        c = _crs(_sub(list(X[1]), list(X[0])), _sub(list(X[3]), list(X[2])))
        cc = _dt(c, c)
        if cc < eps:
            xx = cc / eps
            return (2.0 - xx) * xx * B0
    return B0


def _ccd_d2(X, is_ee, xi):
    d2 = _pair_d2(X, is_ee)
    if is_ee and d2 - xi * xi <= 0:
        # (nearly) parallel edges far apart: the closest endpoint pair
        d2 = min(_d2_pp(list(X[a]), list(X[b])) for a, b in ((0, 2), (0, 3), (1, 2), (1, 3)))
    return d2


def ccd_broadphase(X, dX, is_ee, dist):
    """Swept AABBs of the two sides (point | triangle, edge | edge) over the
    step, apart by more than dist on some axis -> no contact possible
    (collision_detection/filters/lbvh_simplex_trajectory_filter.cu:905-918,
    utils/distance/details/ccd.inl point_triangle_ccd_broadphase)."""
    X = np.asarray(X, dtype=np.float64).reshape(4, 3)
    Y = X + np.asarray(dX, dtype=np.float64).reshape(4, 3)
    a = [0, 1] if is_ee else [0]
    b = [2, 3] if is_ee else [1, 2, 3]
    pa = np.concatenate([X[a], Y[a]])
    pb = np.concatenate([X[b], Y[b]])
    return not (((pa.min(0) - pb.max(0)) > dist).any() or ((pb.min(0) - pa.max(0)) > dist).any())


def accd_toi(X, dX, is_ee, eta=0.1, thickness=0.0, max_iter=1000, toi_max=1.1):
    """(hit, toi) of one pair moving by dX over the step: additive CCD
    (conservative advancement on the pair's distance, Li et al., Codimensional
    Incremental Potential Contact, 2021), as the reference's trajectory
    filter runs it (utils/distance/details/ccd.inl: point_triangle_ccd,
    edge_edge_ccd; filters/lbvh_simplex_trajectory_filter.cu:876-1010):
    the pair's mean displacement removed, l = the largest displacement of
    each side summed, every step advances by (1 - eta) (d^2 - xi^2) /
    ((d + xi) l), the loop ends when the distance function falls below
    eta times its start (after the first step) -- hit at the time reached --
    or when the time passes toi_max (no hit). Written step for step in the
    library's own order of operations (mean over the pair's four vertices
    in order)."""
    X = [list(map(float, r)) for r in np.asarray(X, dtype=np.float64).reshape(4, 3)]
    dX = [list(map(float, r)) for r in np.asarray(dX, dtype=np.float64).reshape(4, 3)]
    mov = [(((dX[0][c] + dX[1][c]) + dX[2][c]) + dX[3][c]) / 4.0 for c in range(3)]
    dX = [[r[c] - mov[c] for c in range(3)] for r in dX]
    n2 = [_dt(r, r) for r in dX]
    if is_ee:
        l = np.sqrt(max(n2[0], n2[1])) + np.sqrt(max(n2[2], n2[3]))
    else:
        l = np.sqrt(n2[0]) + np.sqrt(max(n2[1], n2[2], n2[3]))
    if not (l > 0):
        return False, toi_max
    xi2 = thickness * thickness
    d2 = _ccd_d2(np.array(X), is_ee, thickness)
    f = d2 - xi2
    d = np.sqrt(d2)
    gap = eta * f / (d + thickness)
    t = 0.0
    while True:
        if max_iter <= 0:
            return True, t
        max_iter -= 1
        tl = (1.0 - eta) * f / ((d + thickness) * l)
        X = [[X[i][c] + tl * dX[i][c] for c in range(3)] for i in range(4)]
        d2 = _ccd_d2(np.array(X), is_ee, thickness)
        f = d2 - xi2
        d = np.sqrt(d2)
        if t > 0 and f / (d + thickness) < gap:
            return True, t
        t += tl
        if t > toi_max:
            return False, toi_max


def candidate_pairs(x, dx, alpha, surf_verts, surf_edges, surf_tris, dist):
    """Every candidate pair of the step, by brute force: point-triangle
    (surface vertex, surface triangle) and edge-edge (surface edges i < j)
    whose swept boxes over x -> x + alpha dx are not apart by more than dist
    on any axis (the far test of utils/distance/details/ccd.inl
    point_triangle_ccd_broadphase / edge_edge_ccd_broadphase), pairs sharing
    a vertex excluded. Returns the set of (p, t0, t1, t2) and of
    (a0, a1, b0, b1) tuples."""
    x = np.asarray(x, dtype=np.float64).reshape(-1, 3)
    y = x + alpha * np.asarray(dx, dtype=np.float64).reshape(-1, 3)
    lo, hi = np.minimum(x, y), np.maximum(x, y)
    V = np.asarray(surf_verts).reshape(-1)
    E = np.asarray(surf_edges).reshape(-1, 2)
    T = np.asarray(surf_tris).reshape(-1, 3)

    def boxes(P):
        return lo[P].min(axis=1), hi[P].max(axis=1)

    def near(alo, ahi, blo, bhi):
        far = ((alo[:, None, :] - bhi[None, :, :]) > dist) | ((blo[None, :, :] - ahi[:, None, :]) > dist)
        return ~far.any(axis=2)

    pt = set()
    if len(V) and len(T):
        tlo, thi = boxes(T)
        ok = near(lo[V], hi[V], tlo, thi)
        for i, j in zip(*np.nonzero(ok)):
            v, t = int(V[i]), tuple(int(c) for c in T[j])
            if v not in t:
                pt.add((v,) + t)
    ee = set()
    if len(E) > 1:
        elo, ehi = boxes(E)
        ok = near(elo, ehi, elo, ehi)
        for i, j in zip(*np.nonzero(np.triu(ok, 1))):
            a, b = tuple(int(c) for c in E[i]), tuple(int(c) for c in E[j])
            if not set(a) & set(b):
                ee.add(a + b)
    return pt, ee


def pairs_toi(x, dx, pairs, is_ee, alpha, dhat, thickness=0.0, eta=0.1):
    """The trajectory filter's step bound over a candidate list: per pair the
    broadphase (expanded by dhat + thickness) and the additive CCD of
    alpha dx, 1.1 for pairs without a hit; min(1, the smallest)
    (collision_detection/global_trajectory_filter.cu:111-134)."""
    x = np.asarray(x, dtype=np.float64).reshape(-1, 3)
    dx = alpha * np.asarray(dx, dtype=np.float64).reshape(-1, 3)
    best = 1.1
    for p, ee in zip(np.asarray(pairs).reshape(-1, 4), is_ee):
        X, dX = x[p], dx[p]
        if not ccd_broadphase(X, dX, ee, dhat + thickness):
            continue
        hit, t = accd_toi(X, dX, ee, eta=eta, thickness=thickness)
        if hit:
            best = min(best, t)
    return min(best, 1.0)


# ---- tet-mesh energy (the line search's) ------------------------------------------
def tet_energy(rest, tets, x, x_tilde, mu, lam, rho, dt, ground=None, ground_y=0.0, dhat=1e-3, kappa=1e9):
    """Kinetic (lumped mass rho V / 4 per corner) + dt^2 V Psi_SNH (Psi = mu/2
    (|F|^2 - 3) - mu (J - 1) + lambda/2 (J - 1)^2, the simplified stable
    Neo-Hookean of finite_element/constitutions/sym/simplified_stable_neo_hookean_3d.inl)
    + dt^2 kappa b(d^2) of the ground candidates (b(D) = -(D - Dh)^2 log(D/Dh)),
    in numpy (FP64, numpy's summation order)."""
    rest = np.asarray(rest).reshape(-1, 3)
    x = np.asarray(x).reshape(-1, 3)
    xt = np.asarray(x_tilde).reshape(-1, 3)
    T = np.asarray(tets)
    Dm = np.stack([rest[T[:, q]] - rest[T[:, 0]] for q in (1, 2, 3)], axis=2)
    vol = np.linalg.det(Dm) / 6.0
    Ds = np.stack([x[T[:, q]] - x[T[:, 0]] for q in (1, 2, 3)], axis=2)
    F = Ds @ np.linalg.inv(Dm)
    J = np.linalg.det(F)
    psi = 0.5 * mu * ((F * F).sum(axis=(1, 2)) - 3) - mu * (J - 1) + 0.5 * lam * (J - 1) ** 2
    mass = np.zeros(len(x))
    np.add.at(mass, T.reshape(-1), np.repeat(rho * vol / 4.0, 4))
    e = 0.5 * (mass * ((x - xt) ** 2).sum(1)).sum() + dt * dt * (vol * psi).sum()
    if ground is not None:
        d = x[np.asarray(ground), 1] - ground_y
        if (d <= 0).any():
            return np.inf
        a = d < dhat
        D, Dh = d[a] ** 2, dhat * dhat
        e += dt * dt * kappa * (-(D - Dh) ** 2 * np.log(D / Dh)).sum()
    return float(e)
