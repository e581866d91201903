"""Replica coordination (libuipc_b200/replicas.py) on CPU: two ranks over gloo
(world size 2, rendezvous on 127.0.0.1) agree on the slowest rank's time and on
the units all ranks processed; a single process needs no process group."""
import os
import socket

import pytest


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import torch

    from libuipc_b200.replicas import Replicas

    r = Replicas("gloo", torch.device("cpu"), timeout_s=60)
    r.barrier()
    slowest = r.max(1.5 + rank)  # this rank's "step time"
    units = r.sum(10.0 * (rank + 1))  # this rank's processed units
    r.barrier()
    r.close()
    q.put((rank, slowest, units))


def test_two_gloo_replicas():
    import torch.multiprocessing as mp

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs)
    out = sorted(q.get(timeout=10) for _ in range(world))
    assert [o[0] for o in out] == [0, 1]
    assert all(o[1] == 2.5 for o in out)
    assert all(o[2] == 30.0 for o in out)


def test_single_process_needs_no_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from libuipc_b200.replicas import Replicas

    r = Replicas("gloo", None)
    assert (r.rank, r.world, r.dist) == (0, 1, None)
    r.barrier()
    assert r.max(3.25) == 3.25 and r.sum(7.0) == 7.0
    r.close()
