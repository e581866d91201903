"""Synthetic Newton systems for the linear-solve workloads (host C++ generator).

The generator lives in ``csrc/scene/scene_gen.cpp``; this module only wraps it.
A system holds the raw, unsummed block-upper triplets of one Newton step in
libuipc's conventions (3x3 blocks, column-major values, row <= col), the
gradient ``b`` and the tetrahedral vertex adjacency the MAS partition uses.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._native import load_scene_lib


class B2GConfig(C.Structure):
    _fields_ = [
        ("scene", C.c_int),
        ("cells_x", C.c_int),
        ("cells_y", C.c_int),
        ("cells_z", C.c_int),
        ("n_cubes", C.c_int),
        ("h", C.c_double),
        ("jitter", C.c_double),
        ("normal_jitter", C.c_double),
        ("gap", C.c_double),
        ("seed", C.c_uint64),
        ("E", C.c_double),
        ("nu", C.c_double),
        ("rho", C.c_double),
        ("dt", C.c_double),
        ("gravity", C.c_double),
        ("dhat", C.c_double),
        ("kappa", C.c_double),
        ("ground_offset", C.c_double),
        ("twist_deg", C.c_double),
        ("n_threads", C.c_int),
        ("body_kappa", C.c_double),
        ("bend_k", C.c_double),
        ("cloth_size", C.c_double),
        ("wall_gap", C.c_double),
        ("cloth_n", C.c_int),
        ("bodies_x", C.c_int),
        ("bodies_z", C.c_int),
        ("cloth_k", C.c_double),
    ]


@dataclass
class NewtonSystem:
    """One assembled-but-unreduced Newton system (host arrays)."""

    n_verts: int
    rows: np.ndarray  # int32 [T]
    cols: np.ndarray  # int32 [T]
    vals: np.ndarray  # float64 [T, 9] column-major 3x3 blocks
    b: np.ndarray  # float64 [3 n_verts]
    positions: np.ndarray  # float64 [n_verts, 3]
    tets: np.ndarray  # int32 [n_tets, 4]
    adj_start: np.ndarray  # int32 [n_verts + 1]
    adj_list: np.ndarray  # int32 [nnz]
    n_contacts: int = 0
    config: dict = field(default_factory=dict)
    n_bodies: int = 0  # affine bodies (4 block rows each, first in the DoF order)

    @property
    def n_triplets(self) -> int:
        return int(self.rows.shape[0])

    @property
    def n_dof(self) -> int:
        return 3 * self.n_verts


def default_config() -> B2GConfig:
    lib = load_scene_lib()
    cfg = B2GConfig()
    lib.b2g_default_config(C.byref(cfg))
    return cfg


def _config(overrides: dict) -> B2GConfig:
    cfg = default_config()
    for k, v in overrides.items():
        if not hasattr(cfg, k):
            raise KeyError(f"unknown generator option {k!r}")
        setattr(cfg, k, v)
    return cfg


def generate(**overrides) -> NewtonSystem:
    """Generate a Newton system; keyword arguments override the defaults
    (10x10x10 Kuhn-split cube, E=1e5, nu=0.45, rho=1e3, dt=0.01, dhat=1e-3)."""
    return _generate(_config(overrides), None, None)


def generate_state(x: np.ndarray, x_tilde: np.ndarray, **overrides) -> NewtonSystem:
    """The Newton system of the configured mesh at positions ``x`` with the
    kinetic target ``x_tilde = x_prev + dt v + dt^2 g`` (both ``[n_verts, 3]``).
    The ground stays where the rest shape puts it; the twisted bar's end
    layers are fixed at the positions ``x`` gives them."""
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    xt = np.ascontiguousarray(x_tilde, dtype=np.float64).reshape(-1)
    if x.shape != xt.shape:
        raise ValueError("x and x_tilde differ in size")
    return _generate(_config(overrides), x, xt)


def _generate(cfg: B2GConfig, x, xt) -> NewtonSystem:
    lib = load_scene_lib()
    handle = C.c_void_p()
    if x is None:
        rc = lib.b2g_generate(C.byref(cfg), C.byref(handle))
    else:
        dp = C.POINTER(C.c_double)
        rc = lib.b2g_generate_state(C.byref(cfg), x.ctypes.data_as(dp), xt.ctypes.data_as(dp), C.byref(handle))
    if rc != 0:
        raise RuntimeError("scene generator failed: " + lib.b2g_last_error().decode())
    try:
        nv = lib.b2g_num_verts(handle)
        if x is not None and x.size != 3 * nv:
            raise ValueError(f"state has {x.size // 3} vertices, the mesh {nv}")
        nt = lib.b2g_num_tets(handle)
        T = lib.b2g_num_triplets(handle)
        nadj = lib.b2g_num_adjacency(handle)

        def arr(ptr, n, dtype):
            if n == 0:
                return np.zeros(0, dtype=dtype)
            return np.ctypeslib.as_array(ptr, shape=(n,)).copy()

        sysm = NewtonSystem(
            n_verts=int(nv),
            rows=arr(lib.b2g_triplet_rows(handle), T, np.int32),
            cols=arr(lib.b2g_triplet_cols(handle), T, np.int32),
            vals=arr(lib.b2g_triplet_vals(handle), T * 9, np.float64).reshape(T, 9),
            b=arr(lib.b2g_gradient(handle), nv * 3, np.float64),
            positions=arr(lib.b2g_positions(handle), nv * 3, np.float64).reshape(nv, 3),
            tets=arr(lib.b2g_tets(handle), nt * 4, np.int32).reshape(nt, 4),
            adj_start=arr(lib.b2g_adjacency_start(handle), nv + 1, np.int32),
            adj_list=arr(lib.b2g_adjacency_list(handle), nadj, np.int32),
            n_contacts=int(lib.b2g_num_contacts(handle)),
            config={k: getattr(cfg, k) for k, _ in B2GConfig._fields_},
            n_bodies=int(lib.b2g_num_bodies(handle)),
        )
    finally:
        lib.b2g_free(handle)
    return sysm


def cube_on_ground(cells: int = 10, seed: int = 0, **kw) -> NewtonSystem:
    """Jittered Kuhn-split tet cube resting on a ground plane (one Newton
    system of frame 1 from rest)."""
    return generate(scene=1, cells_x=cells, cells_y=cells, cells_z=cells, n_cubes=1, seed=seed, **kw)


def stacked_cubes(cells: int = 40, n_cubes: int = 8, seed: int = 0, **kw) -> NewtonSystem:
    """``n_cubes`` jittered tet cubes stacked along +y with 1 mm nominal gaps;
    point-triangle / edge-edge barrier blocks couple neighbouring cubes."""
    return generate(scene=1, cells_x=cells, cells_y=cells, cells_z=cells, n_cubes=n_cubes, seed=seed, **kw)


def twisted_bar(nx: int = 200, ny: int = 20, nz: int = 20, twist_deg: float = 2.0, seed: int = 0, **kw) -> NewtonSystem:
    """Bar along x with both end layers fixed and rotated by +-twist_deg."""
    kw.setdefault("E", 1e6)
    kw.setdefault("nu", 0.49)
    return generate(scene=2, cells_x=nx, cells_y=ny, cells_z=nz, n_cubes=1, twist_deg=twist_deg, seed=seed, **kw)


def cloth_on_bodies(n: int = 256, bodies_per_side: int = 8, seed: int = 0, **kw) -> NewtonSystem:
    """n x n-vertex cloth (1 mm sheet, stretch stiffness E, bending bend_k)
    resting on bodies_per_side^2 affine bodies (cubes rotated about +y from
    the seed, orthogonality stiffness body_kappa): 3x3 cloth blocks, 12x12
    body blocks (as 16 3x3 triplets) and 12x3 cloth-body contact couplings.
    The bodies' 4 * n_bodies block rows come first."""
    kw.setdefault("E", 1e3)
    return generate(scene=3, cells_x=n, cells_y=1, cells_z=1, n_cubes=bodies_per_side, seed=seed, **kw)


def cube_wall(cells: int = 30, side: int = 10, cloth_n: int = 512, bodies_x: int = 4, bodies_z: int = 8,
              seed: int = 0, **kw) -> NewtonSystem:
    """The full-scale case: a side x side grid of jittered tet cubes of
    cells^3 cells on the ground (2 cm apart), a cloth_n x cloth_n cloth resting
    on their top faces (point-triangle barrier blocks) and bodies_x x bodies_z
    affine bodies resting on the cloth (12x3 couplings); dt = 5 ms. The
    bodies' 4 * n_bodies block rows come first, then the cube vertices, then
    the cloth; the MAS range is everything after the bodies. The defaults give
    3.26 M block rows (9.8 M DoF)."""
    kw.setdefault("dt", 0.005)
    return generate(scene=4, cells_x=cells, cells_y=cells, cells_z=cells, n_cubes=side, cloth_n=cloth_n,
                    bodies_x=bodies_x, bodies_z=bodies_z, seed=seed, **kw)
