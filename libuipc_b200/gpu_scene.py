"""Newton systems of tet meshes generated on the GPU (include/b200gen.h,
csrc/b2s_generate.cu): kinetic + stable Neo-Hookean (PSD-projected) + ground
barrier + Dirichlet vertices, written straight into device triplet buffers
that :meth:`Solver.assemble` takes. The mesh (rest shape, tets) comes from the
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

    def close(self):
        if self.h:
            _lib().b2gen_mesh_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
