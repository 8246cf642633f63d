"""Replica plumbing of the benchmark on two host processes (gloo): barrier,
maximum and sum over ranks, and the whole-job rate the benchmark reports
(all ranks' particles over the slowest rank's time)."""
import os
import socket

import numpy as np
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
    gathered = rep.gather({"rank": rank, "particles": particles})
    q.put((rank, rep.max(rank * 3.0), rep.sum(rank + 1), rate, ms_max, rep.world, gathered))
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
    for rank, mx, sm, rate, ms_max, w, gathered in out:
        assert w == world and mx == 3.0 and sm == 3.0 and ms_max == 15.0
        assert rate == pytest.approx((1000 + 2000) * 100 / 0.015)
        assert gathered == [{"rank": 0, "particles": 1000}, {"rank": 1, "particles": 2000}]


def test_single_rank_needs_no_process_group(monkeypatch):
    for v in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(v, raising=False)
    from ultraballpit_b200.replicas import Replicas
    rep = Replicas("gloo")
    assert rep.dist is None and rep.world == 1
    assert rep.whole_job_rate(500, 10, 2.0) == (500 * 10 / 0.002, 2.0)
    rep.close()


def test_partition_lpt_balances_and_covers():
    """Greedy bin-packing of instance sizes onto GPUs: every instance exactly
    once, deterministic, and the largest load within the largest instance of
    the mean (the LPT bound)."""
    from ultraballpit_b200.replicas import partition_lpt
    rng = np.random.default_rng(3)
    sizes = np.exp(rng.uniform(np.log(2e3), np.log(4e5), 256)).astype(int).tolist()
    for parts in (1, 2, 3, 8):
        out = partition_lpt(sizes, parts)
        assert out == partition_lpt(sizes, parts)
        assert sorted(i for o in out for i in o) == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in o) for o in out]
        assert max(loads) <= sum(sizes) / parts + max(sizes)
        assert all(o == sorted(o) for o in out)
    assert partition_lpt([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]  # ties go to the lower GPU index
    assert partition_lpt([], 2) == [[], []]
    with pytest.raises(ValueError):
        partition_lpt([1], 0)
