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
    run (and labels the training samples)."""

    def __init__(self, solver: Solver, seq: SceneSequence, device, truth_tol: float = 1e-10):
        import torch

        self.torch = torch
        self.s = solver
        self.seq = seq
        self.dev = device
        self.truth_tol = truth_tol
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
            d = self.history.setdefault(k, deque(maxlen=_abi.B2S_WS_HISTORY))
            d.appendleft(x)
            return x.cpu().numpy()

        for _ in self.seq.run(n_steps, newton_iters, solve):
            pass
        return log
