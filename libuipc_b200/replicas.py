"""One process per GPU, N independent replicas of the linear solve.

The solve does not shard: a Newton system lives on one GPU (the reference
solves on one device as well), so N ranks run N replicas of the same
workload. The only collectives are the barrier that brackets a timed region
and the reductions of per-rank figures (the slowest rank's time, the units
all ranks processed); there is no data-path exchange. Rank, world size and
local rank come from the environment torchrun sets (RANK, WORLD_SIZE,
LOCAL_RANK, MASTER_ADDR, MASTER_PORT); a single process needs none of them.
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    """Process-group membership of one replica. ``backend``: "nccl" on GPUs,
    "gloo" on CPU; ``device``: where the reduction tensors live (the rank's
    GPU for NCCL, CPU for gloo); ``timeout_s`` bounds every collective so a
    rank that never arrives ends the others' wait with an error."""

    def __init__(self, backend: str = "nccl", device=None, timeout_s: float = 300.0):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.device = device
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist

            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def _sync(self):
        if self.device is not None and getattr(self.device, "type", None) == "cuda":
            import torch

            torch.cuda.synchronize(self.device)

    def barrier(self):
        """All ranks' queued GPU work done, then all ranks here."""
        self._sync()
        if self.dist is not None:
            self.dist.barrier()
        self._sync()

    def _reduce(self, v: float, op) -> float:
        if self.dist is None:
            return float(v)
        import torch

        t = torch.tensor([float(v)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, v: float) -> float:
        """The largest per-rank value (a step time: the slowest replica)."""
        return self._reduce(v, self.dist.ReduceOp.MAX if self.dist else None)

    def sum(self, v: float) -> float:
        """The total over ranks (units all replicas processed)."""
        return self._reduce(v, self.dist.ReduceOp.SUM if self.dist else None)

    def close(self):
        """Leave the group (after a last barrier: no rank exits while another
        still waits in a collective)."""
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
