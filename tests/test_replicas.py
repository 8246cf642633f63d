"""Replica plumbing of the benchmark on two host processes (gloo): barrier,
maximum and sum over ranks, and the whole-job rate the benchmark reports
(all ranks' particles over the slowest rank's time)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, q) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from ultraballpit_b200.replicas import Replicas
    rep = Replicas("gloo", timeout_s=60)
    rep.barrier()
    particles = 1000 * (rank + 1)          # uneven work per rank
    ms = 10.0 + 5.0 * rank                 # the last rank is slowest
    rate, ms_max = rep.whole_job_rate(particles, 100, ms)
    q.put((rank, rep.max(rank * 3.0), rep.sum(rank + 1), rate, ms_max, rep.world))
    rep.close()


def test_two_ranks_reduce_max_and_sum_and_rate():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, sm, rate, ms_max, w in out:
        assert w == world and mx == 3.0 and sm == 3.0 and ms_max == 15.0
        assert rate == pytest.approx((1000 + 2000) * 100 / 0.015)


def test_single_rank_needs_no_process_group(monkeypatch):
    for v in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(v, raising=False)
    from ultraballpit_b200.replicas import Replicas
    rep = Replicas("gloo")
    assert rep.dist is None and rep.world == 1
    assert rep.whole_job_rate(500, 10, 2.0) == (500 * 10 / 0.002, 2.0)
    rep.close()
