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
time of impact caps the step too. With ``cfl_dhat`` (the reference's
cfl/enable, off by default there too) a step the time of impact cut is
further capped to 0.5 dhat over the largest surface-vertex displacement.
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


def cfl_bound(d, dhat: float, verts=None) -> float:
    """The contact CFL step bound: min(1, 0.5 dhat / max |d_v|) over the
    surface vertices ``verts`` (every vertex when None), 1 when nothing moves
    (contact_system/global_contact_manager.cu:500-541, config cfl/enable).
    ``d`` is a torch tensor or a numpy array of 3 values per vertex."""
    v = d.reshape(-1, 3)
    if verts is not None:
        v = v[verts]
    if v.shape[0] == 0:
        return 1.0
    m = float((v * v).sum(1).max()) ** 0.5
    return 1.0 if m == 0.0 else min(0.5 * dhat / m, 1.0)


def line_search(mesh, x, d, x_tilde, dt: float, velocity_tol: float = 0.05, max_iter: int = 8,
                contacts=None, trajectory=None, cfl_dhat=None, cfl_verts=None) -> LineSearchResult:
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
    if cfl_dhat is not None and toi < 1.0:
        # the reference's experimental CFL filter, only when a time of impact
        # cut the step (engine/advance_ipc.cu:523-527)
        alpha = min(alpha, cfl_bound(d, cfl_dhat, cfl_verts))
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
