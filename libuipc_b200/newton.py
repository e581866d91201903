"""The step after the solve: the backtracking line search of libuipc's Newton
loop (src/backends/cuda/engine/advance_ipc.cu:487-570), for tet meshes on the
device (`gpu_scene.GpuTetMesh`).

Per Newton iteration: the direction d = -s from the solve of A s = b; the step
starts at alpha = 1, is capped by the ground's time of impact (the vertex /
half-plane trajectory filter, 90 % of the time of impact), then halved until
the energy does not increase (E(x + alpha d) <= E(x)), at most ``max_iter``
times; the state ends at the last trial. An iteration counts as converged
when the largest displacement component of d is at most velocity_tol * dt
(newton/velocity_tol, 0.05 m/s: newton_tolerance/max_translation_checker.cu:43-62)
and the time of impact did not cut the step (newton/ccd_tol = 1); a converged
iteration takes its first trial without the energy test, as the reference does
against rounding-level energy increases from a tiny d. With ``contacts`` (a
`gpu_scene.GpuContacts` set of point-triangle / edge-edge pairs over the same
vertices) the energy adds the pairs' barrier and the step is also capped by
the pairs' continuous collision detection (the simplex trajectory filter:
additive CCD per pair, min(1, the smallest time of impact)); the candidate
pairs are the caller's. With ``trajectory`` (a `gpu_scene.GpuTrajectory` over
the mesh's surface) the candidates of the step are found on the device first
(a hashed uniform grid in place of the reference's BVH) and their smallest
time of impact caps the step too.
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass
class LineSearchResult:
    alpha: float
    toi_alpha: float
    energy0: float
    energy: float
    trials: int
    converged: bool


def line_search(mesh, x, d, x_tilde, dt: float, velocity_tol: float = 0.05, max_iter: int = 8,
                contacts=None, trajectory=None) -> LineSearchResult:
    """Move the device state ``x`` (in place) along ``d`` as the reference's
    line search does; returns the accepted step, the energies and whether the
    Newton iteration had converged."""
    def energy(state):
        e = mesh.energy(state, x_tilde)
        return e + contacts.energy(state) if contacts is not None else e

    x0 = x.clone()
    e0 = energy(x0)
    toi = mesh.ground_toi(x0, d)
    if contacts is not None:
        toi = min(toi, contacts.toi(x0, d))
    if trajectory is not None:
        toi = min(toi, trajectory.toi(x0, d))
    alpha = min(1.0, toi)
    converged = float(d.abs().max()) <= velocity_tol * dt and toi >= 1.0
    e = e0
    trials = 0
    step = alpha  # the step of the state x holds (the last trial's)
    for trials in range(1, max_iter + 1):
        step = alpha
        x.copy_(x0)
        x.add_(d, alpha=step)
        e = energy(x)
        if converged or e <= e0:
            break
        alpha *= 0.5
    return LineSearchResult(alpha=step, toi_alpha=toi, energy0=e0, energy=e, trials=trials, converged=converged)
