"""Time stepping of the synthetic scenes: the Newton systems along a run.

The learned warm start trains on Newton systems the solver itself generates
along a simulated sequence, and is judged on later systems of the same run.
This module advances a scene with backward-Euler steps: each step sets
``x_tilde = x_prev + dt v + dt^2 g``, runs ``newton_iters`` Newton iterations
(assemble at the current positions, solve ``A s = b``, ``x -= s``, full steps,
no line search) and updates ``v = (x - x_prev) / dt``. In the twisted bar the
two end layers are fixed and rotated by ``+-twist_per_step * step`` degrees
about the bar axis each step.
"""
from __future__ import annotations

import math
from typing import Callable, Iterator

import numpy as np

from .scene import NewtonSystem, generate, generate_state


class SceneSequence:
    """A scene stepped through time. ``cfg``: generator options (``scene``,
    ``cells_*``, material, ``dt`` ...); ``twist_per_step``: end rotation rate
    of the twisted bar [deg / step]."""

    def __init__(self, twist_per_step: float = 2.0, **cfg):
        self.cfg = dict(cfg)
        rest_cfg = dict(cfg)
        if rest_cfg.get("scene", 1) == 2:
            rest_cfg["twist_deg"] = 0.0
        base = generate(**rest_cfg)
        c = base.config
        self.dt = float(c["dt"])
        self.gravity = float(c["gravity"])
        self.scene = int(c["scene"])
        self.twist_per_step = float(twist_per_step)
        self.rest = base.positions.copy()
        self.x = self.rest.copy()
        self.v = np.zeros_like(self.x)
        self.x_prev = self.x.copy()
        self.x_tilde = self.x.copy()
        self.adj_start = base.adj_start
        self.adj_list = base.adj_list
        self.n_verts = base.n_verts
        self.n_bodies = int(base.n_bodies)
        # gravity acts on translations: every vertex row and each affine body's
        # first block row (its centre), not on the rows of its affine matrix
        rows = np.arange(self.n_verts)
        self.gravity_rows = (rows >= 4 * self.n_bodies) | (rows % 4 == 0)
        self.step = 0
        if self.scene == 2:
            xs = self.rest[:, 0]
            self.left = np.isclose(xs, xs.min(), atol=1e-12)
            self.right = np.isclose(xs, xs.max(), atol=1e-12)
            self.axis_y = 0.5 * (self.rest[:, 1].min() + self.rest[:, 1].max())
            self.axis_z = 0.5 * (self.rest[:, 2].min() + self.rest[:, 2].max())
        else:
            self.left = self.right = np.zeros(self.n_verts, bool)

    @property
    def fixed(self) -> np.ndarray:
        return self.left | self.right

    def _rotated_rest(self, mask: np.ndarray, deg: float) -> np.ndarray:
        th = math.radians(deg)
        cs, sn = math.cos(th), math.sin(th)
        p = self.rest[mask]
        y, z = p[:, 1] - self.axis_y, p[:, 2] - self.axis_z
        out = p.copy()
        out[:, 1] = self.axis_y + cs * y - sn * z
        out[:, 2] = self.axis_z + sn * y + cs * z
        return out

    def begin_step(self) -> None:
        self.step += 1
        self.x_prev = self.x.copy()
        self.x_tilde = self.x + self.dt * self.v
        self.x_tilde[self.gravity_rows, 1] -= self.dt * self.dt * self.gravity
        if self.scene == 2:
            th = self.twist_per_step * self.step
            self.x[self.left] = self._rotated_rest(self.left, -th)
            self.x[self.right] = self._rotated_rest(self.right, th)

    def system(self) -> NewtonSystem:
        """The Newton system at the current iterate."""
        return generate_state(self.x, self.x_tilde, **self.cfg)

    def apply(self, sol: np.ndarray) -> None:
        """Newton update with the solution of ``A s = b`` (dx = -s)."""
        self.x -= np.asarray(sol, dtype=np.float64).reshape(-1, 3)

    def end_step(self) -> None:
        self.v = (self.x - self.x_prev) / self.dt

    def run(self, n_steps: int, newton_iters: int,
            solve: Callable[[NewtonSystem, int, int], np.ndarray]) -> Iterator[tuple[int, int, NewtonSystem, np.ndarray]]:
        """Step ``n_steps`` times with ``newton_iters`` Newton iterations each;
        ``solve(system, step, k)`` returns ``s`` with ``A s = b``. Yields
        ``(step, k, system, s)`` after each solve."""
        for _ in range(n_steps):
            self.begin_step()
            for k in range(newton_iters):
                sysm = self.system()
                sol = solve(sysm, self.step, k)
                yield self.step, k, sysm, sol
                self.apply(sol)
            self.end_step()


class GpuBarSequence:
    """The twisted bar stepped on the GPU: the state (x, v) stays on the
    device and every Newton system comes from the device generator
    (``gpu_scene.GpuTetMesh``), so a run of thousands of systems needs no host
    work per system. Same stepping as :class:`SceneSequence` (backward Euler,
    end layers fixed and turned by +-twist_per_step * step degrees).
    ``cfg``: generator options of the bar (``cells_*``, material, ``dt``)."""

    def __init__(self, device, twist_per_step: float = 2.0, **cfg):
        import torch

        from .gpu_scene import GpuTetMesh

        self.torch = torch
        self.dev = device
        self.cfg = dict(cfg)
        base = generate(**{**cfg, "scene": 2, "twist_deg": 0.0})
        c = base.config
        self.dt = float(c["dt"])
        self.gravity = float(c["gravity"])
        self.twist_per_step = float(twist_per_step)
        self.rest = base.positions.copy()
        self.n_verts = base.n_verts
        self.adj_start = base.adj_start
        self.adj_list = base.adj_list
        xs = self.rest[:, 0]
        self.left = np.isclose(xs, xs.min(), atol=1e-12)
        self.right = np.isclose(xs, xs.max(), atol=1e-12)
        self.axis_y = 0.5 * (self.rest[:, 1].min() + self.rest[:, 1].max())
        self.axis_z = 0.5 * (self.rest[:, 2].min() + self.rest[:, 2].max())
        self.mesh = GpuTetMesh(self.rest, base.tets, c, device, fixed=self.left | self.right)
        self.x = torch.from_numpy(self.rest.ravel().copy()).to(device)
        self.v = torch.zeros_like(self.x)
        self.x_prev = self.x.clone()
        self.x_tilde = self.x.clone()
        self.fixed_idx = torch.from_numpy(np.nonzero(self.left | self.right)[0]).to(device)
        self.step = 0

    def _turned_ends(self) -> np.ndarray:
        th_deg = self.twist_per_step * self.step
        out = self.rest.copy()
        for mask, sign in ((self.left, -1.0), (self.right, 1.0)):
            th = math.radians(sign * th_deg)
            cs, sn = math.cos(th), math.sin(th)
            y, z = self.rest[mask, 1] - self.axis_y, self.rest[mask, 2] - self.axis_z
            out[mask, 1] = self.axis_y + cs * y - sn * z
            out[mask, 2] = self.axis_z + sn * y + cs * z
        return out[self.left | self.right]

    def begin_step(self) -> None:
        self.step += 1
        self.x_prev = self.x.clone()
        self.x_tilde = self.x + self.dt * self.v
        self.x_tilde.view(-1, 3)[:, 1] -= self.dt * self.dt * self.gravity
        ends = self.torch.from_numpy(self._turned_ends()).to(self.dev)
        self.x.view(-1, 3)[self.fixed_idx] = ends

    def system(self):
        """(rows, cols, vals, b) device tensors of the Newton system at x."""
        return self.mesh.system(self.x, self.x_tilde)

    def apply(self, sol) -> None:
        self.x -= sol

    def end_step(self) -> None:
        self.v = (self.x - self.x_prev) / self.dt

    def close(self) -> None:
        self.mesh.close()
