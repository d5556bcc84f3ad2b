"""Replica plumbing of multi-GPU runs, with two gloo ranks on CPU: each rank
gets its own seed, the barrier holds, and timings reduce to the max over
ranks (the slowest replica sets the job's time)."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from lbm_b200.replicas import Replicas

    reps = Replicas("gloo", timeout_s=60)
    seed = reps.seed(12345)
    reps.barrier()
    ms = reps.max([10.0 + rank, 100.0 - rank])
    q.put((rank, seed, ms))
    reps.close()


def test_two_gloo_replicas_reduce_timings_to_the_max():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [12345, 12346]
    for _, _, ms in got:
        assert ms == [11.0, 100.0]


def test_single_process_needs_no_process_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from lbm_b200.replicas import Replicas

    reps = Replicas("gloo")
    assert reps.world == 1 and reps.dist is None
    assert reps.max([3.0, 4.0]) == [3.0, 4.0]
    reps.close()
