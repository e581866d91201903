"""Newton systems generated on the GPU (include/b200gen.h): tet meshes
(csrc/b2s_generate.cu: kinetic + stable Neo-Hookean (PSD-projected) + ground
barrier + Dirichlet vertices), cloth (csrc/b2s_generate_shell.cu: kinetic +
Baraff-Witkin + discrete-shell bending) and affine bodies (kinetic +
orthogonality potential), written straight into device triplet buffers that
:meth:`Solver.assemble` takes. The mesh (rest shape, tets) comes from the
host generator; only the per-state work runs on the device, so a run of
thousands of Newton systems (the learned warm start's training runs) needs no
host round trip per system.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._native import load_solve_lib


class GenMaterial(C.Structure):
    _fields_ = [("mu", C.c_double), ("lambda_", C.c_double), ("rho", C.c_double), ("dt", C.c_double),
                ("kappa", C.c_double), ("dhat", C.c_double), ("ground_y", C.c_double)]


class ShellMaterial(C.Structure):
    _fields_ = [("stretch", C.c_double), ("shear", C.c_double), ("strain_rate", C.c_double), ("bend", C.c_double),
                ("dt", C.c_double)]


def _lib():
    lib = load_solve_lib()
    if not getattr(lib, "_b2gen_declared", False):
        vp = C.c_void_p
        lib.b2gen_mesh_create.argtypes = [C.c_int, C.c_int32, C.c_int32, vp, vp, vp, C.c_int32, vp,
                                          C.POINTER(GenMaterial), C.POINTER(vp)]
        lib.b2gen_mesh_create.restype = C.c_int
        lib.b2gen_mesh_destroy.argtypes = [vp]
        lib.b2gen_mesh_destroy.restype = C.c_int
        lib.b2gen_num_triplets.argtypes = [vp]
        lib.b2gen_num_triplets.restype = C.c_int64
        lib.b2gen_system.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
        lib.b2gen_system.restype = C.c_int
        lib.b2gen_last_error.argtypes = []
        lib.b2gen_last_error.restype = C.c_char_p
        lib.b2gen_energy.argtypes = [vp, vp, vp, C.POINTER(C.c_double), vp]
        lib.b2gen_energy.restype = C.c_int
        lib.b2gen_ground_toi.argtypes = [vp, vp, vp, C.POINTER(C.c_double), vp]
        lib.b2gen_ground_toi.restype = C.c_int
        i32 = C.c_int32
        lib.b2gen_shell_create.argtypes = [C.c_int, i32, i32, vp, vp, vp, vp, C.POINTER(ShellMaterial),
                                           C.POINTER(vp)]
        lib.b2gen_shell_create.restype = C.c_int
        lib.b2gen_shell_destroy.argtypes = [vp]
        lib.b2gen_shell_destroy.restype = C.c_int
        lib.b2gen_shell_num_triplets.argtypes = [vp]
        lib.b2gen_shell_num_triplets.restype = C.c_int64
        lib.b2gen_shell_num_hinges.argtypes = [vp]
        lib.b2gen_shell_num_hinges.restype = i32
        lib.b2gen_shell_system.argtypes = [vp, vp, vp, i32, vp, vp, vp, vp, vp]
        lib.b2gen_shell_system.restype = C.c_int
        lib.b2gen_abd_create.argtypes = [C.c_int, i32, vp, vp, vp, C.c_double, C.POINTER(vp)]
        lib.b2gen_abd_create.restype = C.c_int
        lib.b2gen_abd_destroy.argtypes = [vp]
        lib.b2gen_abd_destroy.restype = C.c_int
        lib.b2gen_abd_system.argtypes = [vp, vp, vp, i32, vp, vp, vp, vp, vp]
        lib.b2gen_abd_system.restype = C.c_int
        lib.b2gen_contacts_create.argtypes = [C.c_int, i32, vp, vp, vp, C.c_double, C.c_double, C.c_double,
                                              C.POINTER(vp)]
        lib.b2gen_contacts_create.restype = C.c_int
        lib.b2gen_contacts_destroy.argtypes = [vp]
        lib.b2gen_contacts_destroy.restype = C.c_int
        lib.b2gen_contacts_types.argtypes = [vp, vp]
        lib.b2gen_contacts_types.restype = C.c_int
        lib.b2gen_contacts_system.argtypes = [vp, vp, vp, vp, vp, vp, vp]
        lib.b2gen_contacts_system.restype = C.c_int
        lib.b2gen_contacts_energy.argtypes = [vp, vp, C.POINTER(C.c_double), vp]
        lib.b2gen_contacts_energy.restype = C.c_int
        lib.b2gen_contacts_toi.argtypes = [vp, vp, vp, C.c_double, C.POINTER(C.c_double), vp]
        lib.b2gen_contacts_toi.restype = C.c_int
        lib.b2gen_trajectory_create.argtypes = [C.c_int, i32, i32, vp, i32, vp, i32, vp, C.c_double, C.c_double,
                                                C.POINTER(vp)]
        lib.b2gen_trajectory_create.restype = C.c_int
        lib.b2gen_trajectory_destroy.argtypes = [vp]
        lib.b2gen_trajectory_destroy.restype = C.c_int
        lib.b2gen_trajectory_detect.argtypes = [vp, vp, vp, C.c_double, vp, vp]
        lib.b2gen_trajectory_detect.restype = C.c_int
        lib.b2gen_trajectory_pairs.argtypes = [vp, vp, vp]
        lib.b2gen_trajectory_pairs.restype = C.c_int
        lib.b2gen_trajectory_toi.argtypes = [vp, vp, vp, C.c_double, C.POINTER(C.c_double), vp]
        lib.b2gen_trajectory_toi.restype = C.c_int
        lib.b2gen_trajectory_last_error.argtypes = []
        lib.b2gen_trajectory_last_error.restype = C.c_char_p
        lib.b2gen_shell_last_error.argtypes = []
        lib.b2gen_shell_last_error.restype = C.c_char_p
        lib._b2gen_declared = True
    return lib


class GpuTetMesh:
    """A tet mesh on the device. ``rest`` [n, 3], ``tets`` [m, 4]; ``config``:
    the generator settings (E, nu, rho, dt, kappa, dhat); ``fixed``: Dirichlet
    flags [n] or None; ``ground``: candidate vertices of the ground barrier and
    ``ground_y`` its height."""

    def __init__(self, rest, tets, config: dict, device, fixed=None, ground=None, ground_y: float = 0.0):
        import torch

        self.torch = torch
        self.dev = device
        E, nu = float(config["E"]), float(config["nu"])
        mat = GenMaterial(E / (2.0 * (1.0 + nu)), E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), float(config["rho"]),
                          float(config["dt"]), float(config["kappa"]), float(config["dhat"]), float(ground_y))
        rest = np.ascontiguousarray(rest, dtype=np.float64)
        tets = np.ascontiguousarray(tets, dtype=np.int32)
        self.n_verts = rest.shape[0]
        fx = None if fixed is None else np.ascontiguousarray(fixed, dtype=np.uint8)
        gr = None if ground is None else np.ascontiguousarray(ground, dtype=np.int32)
        lib = _lib()
        self.h = C.c_void_p()
        rc = lib.b2gen_mesh_create(device.index or 0, self.n_verts, tets.shape[0], rest.ctypes.data, tets.ctypes.data,
                                   None if fx is None else fx.ctypes.data, 0 if gr is None else len(gr),
                                   None if gr is None else gr.ctypes.data, C.byref(mat), C.byref(self.h))
        if rc != 0:
            raise RuntimeError("b2gen_mesh_create: " + lib.b2gen_last_error().decode())
        self.n_triplets = int(lib.b2gen_num_triplets(self.h))
        T = self.n_triplets
        self.rows = torch.empty(T, dtype=torch.int32, device=device)
        self.cols = torch.empty(T, dtype=torch.int32, device=device)
        self.vals = torch.empty((T, 9), dtype=torch.float64, device=device)
        self.grad = torch.empty(3 * self.n_verts, dtype=torch.float64, device=device)

    def system(self, x, x_tilde, stream=None):
        """The Newton system at device state x, x_tilde ([n*3] float64):
        (rows, cols, vals, b) device tensors (reused between calls)."""
        x = x.contiguous()
        x_tilde = x_tilde.contiguous()
        st = stream if stream is not None else self.torch.cuda.current_stream(self.dev).cuda_stream
        lib = _lib()
        rc = lib.b2gen_system(self.h, x.data_ptr(), x_tilde.data_ptr(), self.rows.data_ptr(), self.cols.data_ptr(),
                              self.vals.data_ptr(), self.grad.data_ptr(), st)
        if rc != 0:
            raise RuntimeError("b2gen_system: " + lib.b2gen_last_error().decode())
        return self.rows, self.cols, self.vals, self.grad

    def system_into(self, x, x_tilde, rows_ptr: int, cols_ptr: int, vals_ptr: int, stream=None):
        """The Newton system written to the given device addresses (e.g. the
        solver-owned triplet arrays of Solver.triplet_buffers); returns b."""
        x = x.contiguous()
        x_tilde = x_tilde.contiguous()
        st = stream if stream is not None else self.torch.cuda.current_stream(self.dev).cuda_stream
        lib = _lib()
        rc = lib.b2gen_system(self.h, x.data_ptr(), x_tilde.data_ptr(), rows_ptr, cols_ptr, vals_ptr,
                              self.grad.data_ptr(), st)
        if rc != 0:
            raise RuntimeError("b2gen_system: " + lib.b2gen_last_error().decode())
        return self.grad

    def energy(self, x, x_tilde, stream=None) -> float:
        """The energy b2gen_system differentiates, at device state x."""
        st = stream if stream is not None else self.torch.cuda.current_stream(self.dev).cuda_stream
        e = C.c_double()
        rc = _lib().b2gen_energy(self.h, x.contiguous().data_ptr(), x_tilde.contiguous().data_ptr(), C.byref(e), st)
        if rc != 0:
            raise RuntimeError("b2gen_energy: " + _lib().b2gen_last_error().decode())
        return float(e.value)

    def ground_toi(self, x, dx, stream=None) -> float:
        """Largest step (<= 1) along dx before a ground candidate reaches the
        plane, with the trajectory filter's 10 % margin."""
        st = stream if stream is not None else self.torch.cuda.current_stream(self.dev).cuda_stream
        a = C.c_double()
        rc = _lib().b2gen_ground_toi(self.h, x.contiguous().data_ptr(), dx.contiguous().data_ptr(), C.byref(a), st)
        if rc != 0:
            raise RuntimeError("b2gen_ground_toi: " + _lib().b2gen_last_error().decode())
        return float(a.value)

    def close(self):
        if self.h:
            _lib().b2gen_mesh_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuShell:
    """A cloth on the device: rest positions [n, 3], triangles [m, 3], lumped
    masses [n]; stretch / shear / strain_rate (Baraff-Witkin), bend (discrete-
    shell bending), dt. Its block rows start at ``vertex_offset`` of the global
    system; :meth:`system_into` writes its triplet slots
    ([n kinetic][6 m triangle blocks][10 per hinge]) and its rows of the global
    gradient."""

    def __init__(self, rest, tris, mass, stretch, shear, bend, dt, device, strain_rate=100.0, fixed=None):
        rest = np.ascontiguousarray(rest, dtype=np.float64)
        tris = np.ascontiguousarray(tris, dtype=np.int32)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        fx = None if fixed is None else np.ascontiguousarray(fixed, dtype=np.uint8)
        mat = ShellMaterial(float(stretch), float(shear), float(strain_rate), float(bend), float(dt))
        self.n_verts = rest.shape[0]
        lib = _lib()
        self.h = C.c_void_p()
        rc = lib.b2gen_shell_create(device.index or 0, self.n_verts, tris.shape[0], rest.ctypes.data,
                                    tris.ctypes.data, mass.ctypes.data, None if fx is None else fx.ctypes.data,
                                    C.byref(mat), C.byref(self.h))
        if rc != 0:
            raise RuntimeError("b2gen_shell_create: " + lib.b2gen_shell_last_error().decode())
        self.n_triplets = int(lib.b2gen_shell_num_triplets(self.h))
        self.n_hinges = int(lib.b2gen_shell_num_hinges(self.h))
        self.dev = device

    def system_into(self, x, x_tilde, vertex_offset, rows_ptr, cols_ptr, vals_ptr, grad, stream=None):
        import torch

        st = stream if stream is not None else torch.cuda.current_stream(self.dev).cuda_stream
        lib = _lib()
        rc = lib.b2gen_shell_system(self.h, x.data_ptr(), x_tilde.data_ptr(), int(vertex_offset), rows_ptr, cols_ptr,
                                    vals_ptr, grad.data_ptr(), st)
        if rc != 0:
            raise RuntimeError("b2gen_shell_system: " + lib.b2gen_shell_last_error().decode())

    def close(self):
        if self.h:
            _lib().b2gen_shell_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuAffineBodies:
    """Affine bodies on the device: mass matrices [nb, 12, 12], orthogonality
    stiffness and volume per body, dt. :meth:`system_into` writes 16 triplets
    per body and the bodies' rows of the global gradient."""

    def __init__(self, mass12, kappa, volume, dt, device):
        M = np.ascontiguousarray(mass12, dtype=np.float64).reshape(-1, 144)
        k = np.ascontiguousarray(kappa, dtype=np.float64)
        v = np.ascontiguousarray(volume, dtype=np.float64)
        self.n_bodies = M.shape[0]
        lib = _lib()
        self.h = C.c_void_p()
        rc = lib.b2gen_abd_create(device.index or 0, self.n_bodies, M.ctypes.data, k.ctypes.data, v.ctypes.data,
                                  float(dt), C.byref(self.h))
        if rc != 0:
            raise RuntimeError("b2gen_abd_create: " + lib.b2gen_shell_last_error().decode())
        self.n_triplets = 16 * self.n_bodies
        self.dev = device

    def system_into(self, q, q_tilde, block_offset, rows_ptr, cols_ptr, vals_ptr, grad, stream=None):
        import torch

        st = stream if stream is not None else torch.cuda.current_stream(self.dev).cuda_stream
        lib = _lib()
        rc = lib.b2gen_abd_system(self.h, q.data_ptr(), q_tilde.data_ptr(), int(block_offset), rows_ptr, cols_ptr,
                                  vals_ptr, grad.data_ptr(), st)
        if rc != 0:
            raise RuntimeError("b2gen_abd_system: " + lib.b2gen_shell_last_error().decode())

    def close(self):
        if self.h:
            _lib().b2gen_abd_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuContacts:
    """Point-triangle / edge-edge contact pairs on the device: pairs [n, 4]
    (global block rows), is_ee [n], eps [n] (edge-edge mollifier thresholds),
    dhat, kappa, dt. :meth:`system_into` writes 10 triplets per pair and adds
    the pairs' gradients to ``grad``."""

    def __init__(self, pairs, is_ee, eps, dhat, kappa, dt, device):
        P = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 4)
        E = np.ascontiguousarray(is_ee, dtype=np.uint8)
        S = np.ascontiguousarray(eps, dtype=np.float64)
        self.n_pairs = P.shape[0]
        lib = _lib()
        self.h = C.c_void_p()
        rc = lib.b2gen_contacts_create(device.index or 0, self.n_pairs, P.ctypes.data, E.ctypes.data, S.ctypes.data,
                                       float(dhat), float(kappa), float(dt), C.byref(self.h))
        if rc != 0:
            raise RuntimeError("b2gen_contacts_create: " + lib.b2gen_shell_last_error().decode())
        self.n_triplets = 10 * self.n_pairs
        self.dev = device

    def system_into(self, x, rows_ptr, cols_ptr, vals_ptr, grad, stream=None):
        import torch

        st = stream if stream is not None else torch.cuda.current_stream(self.dev).cuda_stream
        lib = _lib()
        rc = lib.b2gen_contacts_system(self.h, x.data_ptr(), rows_ptr, cols_ptr, vals_ptr, grad.data_ptr(), st)
        if rc != 0:
            raise RuntimeError("b2gen_contacts_system: " + lib.b2gen_shell_last_error().decode())

    def energy(self, x, stream=None) -> float:
        """The pairs' barrier energy at device state x (the line search's
        contact term), summed in a fixed order."""
        import torch

        st = stream if stream is not None else torch.cuda.current_stream(self.dev).cuda_stream
        e = C.c_double()
        rc = _lib().b2gen_contacts_energy(self.h, x.contiguous().data_ptr(), C.byref(e), st)
        if rc != 0:
            raise RuntimeError("b2gen_contacts_energy: " + _lib().b2gen_shell_last_error().decode())
        return float(e.value)

    def toi(self, x, dx, alpha: float = 1.0, stream=None) -> float:
        """Largest fraction (<= 1) of the move alpha dx from x that the pairs
        allow: additive CCD per pair after a swept-box test."""
        import torch

        st = stream if stream is not None else torch.cuda.current_stream(self.dev).cuda_stream
        t = C.c_double()
        rc = _lib().b2gen_contacts_toi(self.h, x.contiguous().data_ptr(), dx.contiguous().data_ptr(), float(alpha),
                                       C.byref(t), st)
        if rc != 0:
            raise RuntimeError("b2gen_contacts_toi: " + _lib().b2gen_shell_last_error().decode())
        return float(t.value)

    def types(self) -> np.ndarray:
        """Closest-feature type per pair at the last system (0 PP, 1 PE, 2 PT,
        3 EE, -1 beyond dhat)."""
        out = np.zeros(self.n_pairs, np.int8)
        rc = _lib().b2gen_contacts_types(self.h, out.ctypes.data)
        if rc != 0:
            raise RuntimeError("b2gen_contacts_types: " + _lib().b2gen_shell_last_error().decode())
        return out

    def close(self):
        if self.h:
            _lib().b2gen_contacts_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tet_surface(tets):
    """Boundary of a tet mesh (host): the triangles that belong to one tet
    only [m, 3], their edges [e, 2] (each once, smaller id first) and their
    vertices [v], all sorted."""
    T = np.asarray(tets, dtype=np.int64).reshape(-1, 4)
    faces = np.concatenate([T[:, [0, 1, 2]], T[:, [0, 1, 3]], T[:, [0, 2, 3]], T[:, [1, 2, 3]]])
    f = np.sort(faces, axis=1)
    n = int(T.max()) + 1 if T.size else 1
    key = (f[:, 0] * n + f[:, 1]) * n + f[:, 2]  # one int64 per face (n^3 < 2^63 up to 2 M vertices)
    if n >= (1 << 21):
        raise ValueError("tet_surface: more than 2^21 vertices")
    _, idx, cnt = np.unique(key, return_index=True, return_counts=True)
    tris = faces[np.sort(idx[cnt == 1])]
    e = np.sort(np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [0, 2]]]), axis=1)
    ek = np.unique(e[:, 0] * n + e[:, 1])
    edges = np.stack([ek // n, ek % n], axis=1)
    verts = np.unique(tris)
    return tris.astype(np.int32), edges.astype(np.int32), verts.astype(np.int32)


class GpuTrajectory:
    """The line search's trajectory filter over a surface on the device:
    candidate point-triangle / edge-edge pairs of the swept step (a hashed
    uniform grid of cell size ``cell``, pairs within ``dhat``) and the
    smallest time of impact over them (additive CCD)."""

    def __init__(self, n_verts, surf_verts, surf_edges, surf_tris, dhat, cell, device):
        V = np.ascontiguousarray(surf_verts, dtype=np.int32).reshape(-1)
        E = np.ascontiguousarray(surf_edges, dtype=np.int32).reshape(-1, 2)
        T = np.ascontiguousarray(surf_tris, dtype=np.int32).reshape(-1, 3)
        lib = _lib()
        self.h = C.c_void_p()
        rc = lib.b2gen_trajectory_create(device.index or 0, int(n_verts), V.size, V.ctypes.data, E.shape[0],
                                         E.ctypes.data, T.shape[0], T.ctypes.data, float(dhat), float(cell),
                                         C.byref(self.h))
        if rc != 0:
            raise RuntimeError("b2gen_trajectory_create: " + lib.b2gen_trajectory_last_error().decode())
        self.dev = device

    def _stream(self, stream):
        import torch

        return stream if stream is not None else torch.cuda.current_stream(self.dev).cuda_stream

    def detect(self, x, dx, alpha: float = 1.0, stream=None):
        """Candidate pairs [n, 4] and is_ee [n] (point-triangle first) of the
        move alpha dx from x."""
        lib = _lib()
        counts = np.zeros(2, np.int64)
        rc = lib.b2gen_trajectory_detect(self.h, x.contiguous().data_ptr(), dx.contiguous().data_ptr(), float(alpha),
                                         counts.ctypes.data, self._stream(stream))
        if rc != 0:
            raise RuntimeError("b2gen_trajectory_detect: " + lib.b2gen_trajectory_last_error().decode())
        n = int(counts.sum())
        pairs = np.zeros((max(n, 1), 4), np.int32)
        is_ee = np.zeros(max(n, 1), np.uint8)
        rc = lib.b2gen_trajectory_pairs(self.h, pairs.ctypes.data, is_ee.ctypes.data)
        if rc != 0:
            raise RuntimeError("b2gen_trajectory_pairs: " + lib.b2gen_trajectory_last_error().decode())
        return pairs[:n], is_ee[:n]

    def toi(self, x, dx, alpha: float = 1.0, stream=None) -> float:
        """Largest fraction (<= 1) of the move alpha dx from x before a surface
        pair comes into contact."""
        lib = _lib()
        t = C.c_double()
        rc = lib.b2gen_trajectory_toi(self.h, x.contiguous().data_ptr(), dx.contiguous().data_ptr(), float(alpha),
                                      C.byref(t), self._stream(stream))
        if rc != 0:
            raise RuntimeError("b2gen_trajectory_toi: " + lib.b2gen_trajectory_last_error().decode())
        return float(t.value)

    def close(self):
        if self.h:
            _lib().b2gen_trajectory_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
