"""Learned PCG warm start over a simulated run (host orchestration).

The network and its kernels live in csrc/b2s_learned.cu (include/b200solve.h,
b2s_ws_*); this module drives them over a :class:`SceneSequence`: every Newton
system of the run is assembled and solved on the GPU, the solutions are kept
per Newton-iteration index as the history the warm start reads (newest
first), training samples are the systems of the run with their solved x, and
the evaluation solves later systems from each kind of start.
"""
from __future__ import annotations

from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .linear_system import Solver, partition_maps, partition_rcb
from .sequence import SceneSequence

MODES = {
    "zero": _abi.B2S_WS_MODE_ZERO,
    "prev": _abi.B2S_WS_MODE_PREV,
    "history": _abi.B2S_WS_MODE_HISTORY,
    "learned": _abi.B2S_WS_MODE_LEARNED,
}


@dataclass
class SolveRecord:
    step: int
    k: int
    mode: str
    iterations: int
    rel_res: float
    rel_res0: float
    predict_ms: float
    used_mode: int


@dataclass
class RunLog:
    records: list = field(default_factory=list)

    def mean_iterations(self, mode: str, steps=None) -> float:
        its = [r.iterations for r in self.records if r.mode == mode and (steps is None or r.step in steps)]
        return float(np.mean(its)) if its else float("nan")


class SequenceRunner:
    """Solve the Newton systems of ``seq`` with ``solver`` (MAS-PCG on one
    GPU). ``truth_tol``: FP64 relative residual of the solve that advances the
    run (and labels the training samples); ``history``: solutions kept per
    Newton-iteration slot for the starts (at most B2S_WS_MAX_HISTORY; the
    network's fields read the newest 3). A run whose motion is smooth in time
    (a driven twist) gains from a long history, one dominated by contacts
    (a falling stack) from 3 at most."""

    def __init__(self, solver: Solver, seq: SceneSequence, device, truth_tol: float = 1e-10,
                 history: int = _abi.B2S_WS_MAX_HISTORY):
        import torch

        self.torch = torch
        self.s = solver
        self.seq = seq
        self.dev = device
        self.truth_tol = truth_tol
        self.keep = max(1, min(int(history), _abi.B2S_WS_MAX_HISTORY))
        self.p2r, self.r2p = partition_maps(partition_rcb(seq.rest))
        self.s.mas_init(0, seq.n_verts, seq.adj_start, seq.adj_list, self.p2r, self.r2p)
        self.history: dict[int, deque] = {}

    def hist(self, k: int) -> list:
        return list(self.history.get(k, deque()))

    def load(self, sysm):
        """Assemble the system and build the MAS preconditioner; returns b (device)."""
        t = self.torch
        rows = t.from_numpy(sysm.rows).to(self.dev)
        cols = t.from_numpy(sysm.cols).to(self.dev)
        vals = t.from_numpy(np.ascontiguousarray(sysm.vals)).to(self.dev)
        self.s.assemble(sysm.n_verts, rows, cols, vals)
        self.s.precond_assemble(_abi.B2S_PRECOND_MAS)
        return t.from_numpy(sysm.b).to(self.dev)

    def solve_mode(self, b, k: int, mode: str, tol: float = 1e-4, precision=_abi.B2S_PRECISION_FP64,
                   replace_every: int = 50):
        """PCG to FP64-verified rel-res ``tol`` from the start of ``mode``."""
        x = self.torch.zeros_like(b)
        info = self.s.ws_predict(b, x, self.hist(k), MODES[mode])
        st = self.s.pcg(b, x, tol=tol, stop_rule=_abi.B2S_STOP_RELRES, check_interval=5, precision=precision,
                        x0_given=True, replace_every=replace_every)
        return x, st, info

    def run(self, n_steps: int, newton_iters: int = 1, collect: bool = True, eval_modes=(), eval_from: int = 0,
            tol: float = 1e-4, precision=_abi.B2S_PRECISION_FP64) -> RunLog:
        """Advance ``n_steps``; each Newton system is solved to ``truth_tol``
        (FP64, started from the history Galerkin start); with ``collect``
        (after ``ws_init``) its training sample is stored; from
        step ``eval_from`` on, each of ``eval_modes`` is also solved to ``tol``
        and logged."""
        log = RunLog()

        def solve(sysm, step, k):
            b = self.load(sysm)
            if step >= eval_from:
                for mode in eval_modes:
                    _, st, info = self.solve_mode(b, k, mode, tol=tol, precision=precision)
                    log.records.append(SolveRecord(step, k, mode, int(st["iterations_exact"]), float(st["rel_res"]),
                                                   float(info["rel_res0"]), float(info["predict_ms"]),
                                                   int(info["mode"])))
            x = self.torch.zeros_like(b)
            self.s.ws_predict(b, x, self.hist(k), MODES["history"])
            st = self.s.pcg(b, x, tol=self.truth_tol, stop_rule=_abi.B2S_STOP_RELRES, check_interval=5,
                            x0_given=True)
            if collect:
                self.s.ws_add_sample(b, x, self.hist(k))
            d = self.history.setdefault(k, deque(maxlen=self.keep))
            d.appendleft(x)
            return x.cpu().numpy()

        for _ in self.seq.run(n_steps, newton_iters, solve):
            pass
        return log


CHECKPOINT_VERSION = 1


def _hidden_of(n_params: int) -> int:
    """Hidden width from the parameter count (H^2 + 28 H + 4 weights and biases
    plus 2 x 22 feature statistics at 22 features and 4 outputs)."""
    F, O = _abi.B2S_WS_FEATURES, _abi.B2S_WS_OUTPUTS
    for h in range(32, 1025, 32):
        if F * h + h + h * h + h + h * O + O + 2 * F == n_params:
            return h
    raise ValueError(f"no hidden width has {n_params} parameters")


def save_checkpoint(solver: Solver, path: str, with_samples: bool = True) -> None:
    """The learned warm start to an .npz file: format version, hidden width,
    the parameters with the feature statistics (b2s_ws_get_params) and, with
    ``with_samples``, the stored training set (per sample its aggregate rows
    of features, field Gram, q, |x|^2 and its loss normaliser)."""
    params = solver.ws_params()
    out = {"version": np.int32(CHECKPOINT_VERSION), "hidden": np.int32(_hidden_of(params.size)), "params": params}
    if with_samples:
        n, _ = solver.ws_num_samples()
        parts = [solver.ws_sample(i) for i in range(n)]
        out["rows"] = np.array([p["c0"].size for p in parts], np.int64)
        out["norms"] = np.array([p["norm"] for p in parts], np.float64)
        for key in ("feat", "H", "q", "c0"):
            out[key] = (np.concatenate([p[key] for p in parts]) if parts else np.zeros(0, np.float32))
    np.savez(path, **out)


def load_checkpoint(solver: Solver, path: str, with_samples: bool = True) -> int:
    """Restore a checkpoint written by save_checkpoint into ``solver`` (its
    network is created with the stored width); returns the samples appended.
    The optimiser state is not stored: training resumes with fresh moments."""
    d = np.load(path)
    if int(d["version"]) != CHECKPOINT_VERSION:
        raise ValueError(f"checkpoint format {int(d['version'])}, this library reads {CHECKPOINT_VERSION}")
    solver.ws_init(int(d["hidden"]))
    solver.ws_set_params(d["params"])
    if not with_samples or "rows" not in d:
        return 0
    r0 = 0
    for rows, norm in zip(d["rows"], d["norms"]):
        r1 = r0 + int(rows)
        solver.ws_put_sample(d["feat"][r0:r1], d["H"][r0:r1], d["q"][r0:r1], d["c0"][r0:r1], float(norm))
        r0 = r1
    return int(d["rows"].size)


def run_gpu_bar(device, cells=(200, 20, 20), E: float = 1e6, nu: float = 0.49, twist: float = 2.0,
                train_steps: int = 200, eval_steps: int = 20, newton_iters: int = 10, truth_tol: float = 1e-10,
                tol: float = 1e-4, epochs: int = 5, hidden: int = 128, seed: int = 0,
                precision=_abi.B2S_PRECISION_FP64, modes=("zero", "prev", "history", "learned")) -> dict:
    """The learned warm start on a twisted bar at full scale (200x20x20 cells by default): the bar
    (cells, E, nu; ends turned +-twist deg per step) is stepped on the GPU
    (:class:`GpuBarSequence`, every system from the device generator) for
    ``train_steps`` steps of ``newton_iters`` Newton iterations; every system
    is solved to ``truth_tol`` (FP64 MAS-PCG from the history start) and is a
    training sample (train_steps * newton_iters systems); the MLP is trained
    for ``epochs`` epochs; then ``eval_steps`` more steps are run and each of
    their systems is also solved to ``tol`` from every start in ``modes``.
    Returns the mean PCG iterations per mode and the run's timings."""
    import time
    from collections import deque

    import torch

    from .sequence import GpuBarSequence

    seq = GpuBarSequence(device, twist_per_step=twist, cells_x=cells[0], cells_y=cells[1], cells_z=cells[2], E=E,
                         nu=nu)
    solver = Solver(device.index or 0)
    stream = torch.cuda.current_stream(device)
    solver.set_stream(stream.cuda_stream)  # one stream for the solver, the generator and the state updates
    try:
        p2r, r2p = partition_maps(partition_rcb(seq.rest))
        solver.mas_init(0, seq.n_verts, seq.adj_start, seq.adj_list, p2r, r2p)
        solver.ws_init(hidden, seed=seed)
        history: dict[int, deque] = {}
        log = RunLog()
        # timed evaluation: plain FP64 from zero vs mixed precision from the
        # learned start (prediction + PCG, CUDA events; assembly and the MAS
        # build are shared)
        timed = {"plain": ("zero", _abi.B2S_PRECISION_FP64), "mixed+learned": ("learned", _abi.B2S_PRECISION_MIXED)}
        tsum = {k: [0.0, 0, 0] for k in timed}
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def newton(collect: bool, eval_modes) -> None:
            for k in range(newton_iters):
                rows, cols, vals, b = seq.system()
                solver.assemble(seq.n_verts, rows, cols, vals)
                solver.precond_assemble(_abi.B2S_PRECOND_MAS)
                hist = list(history.get(k, deque()))
                if eval_modes:
                    for label, (mode, prec) in timed.items():
                        xm = torch.zeros_like(b)
                        ev0.record(stream)
                        if mode != "zero":
                            solver.ws_predict(b, xm, hist, MODES[mode])
                        st = solver.pcg(b, xm, tol=tol, stop_rule=_abi.B2S_STOP_RELRES, check_interval=5,
                                        precision=prec, x0_given=mode != "zero", replace_every=50)
                        ev1.record(stream)
                        ev1.synchronize()
                        tsum[label][0] += ev0.elapsed_time(ev1)
                        tsum[label][1] += int(st["iterations_exact"])
                        tsum[label][2] += 1
                for mode in eval_modes:
                    xm = torch.zeros_like(b)
                    info = solver.ws_predict(b, xm, hist, MODES[mode])
                    st = solver.pcg(b, xm, tol=tol, stop_rule=_abi.B2S_STOP_RELRES, check_interval=5,
                                    precision=precision, x0_given=True, replace_every=50)
                    log.records.append(SolveRecord(seq.step, k, mode, int(st["iterations_exact"]),
                                                   float(st["rel_res"]), float(info["rel_res0"]),
                                                   float(info["predict_ms"]), int(info["mode"])))
                x = torch.zeros_like(b)
                solver.ws_predict(b, x, hist, MODES["history"])
                solver.pcg(b, x, tol=truth_tol, stop_rule=_abi.B2S_STOP_RELRES, check_interval=5, x0_given=True)
                if collect:
                    solver.ws_add_sample(b, x, hist)
                history.setdefault(k, deque(maxlen=_abi.B2S_WS_MAX_HISTORY)).appendleft(x)
                seq.apply(x)

        t0 = time.time()
        for _ in range(train_steps):
            seq.begin_step()
            newton(True, ())
            seq.end_step()
        stream.synchronize()
        t_run = time.time() - t0
        n_samples, _ = solver.ws_num_samples()
        t0 = time.time()
        solver.ws_fit_normalization()
        loss = solver.ws_train(epochs, lr=1e-3, seed=seed)
        t_train = time.time() - t0
        for _ in range(eval_steps):
            seq.begin_step()
            newton(False, modes)
            seq.end_step()
        return {
            "workload": f"twisted bar {cells[0]}x{cells[1]}x{cells[2]} cells ({seq.n_verts:,} vertices, "
                        f"{3 * seq.n_verts:,} DoF), E={E:g}, nu={nu}, ends +-{twist} deg per step",
            "training_systems": int(n_samples), "train_steps": train_steps, "newton_iters": newton_iters,
            "eval_systems": eval_steps * newton_iters, "epochs": epochs, "final_loss": loss,
            "run_s": t_run, "train_s": t_train,
            "mean_pcg_iterations": {m: log.mean_iterations(m) for m in modes},
            "timed_eval": {k: {"ms_per_solve": v[0] / max(v[2], 1), "mean_pcg_iterations": v[1] / max(v[2], 1),
                               "note": "prediction + PCG; assembly and MAS build shared"}
                           for k, v in tsum.items()},
            "stop": f"rel-res {tol:g}", "precision": "fp64" if precision == _abi.B2S_PRECISION_FP64 else "mixed",
        }
    finally:
        solver.close()
        seq.close()
