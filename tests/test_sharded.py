"""A sharded batch run equals the one-rank run, instance by instance.

Independent simulations shard across GPUs with no exchange on the data path
(each rank takes its share of a greedy bin-packing, ``partition_lpt``) and a
host gather at the end. Two ranks over gloo each run their share of a small
draw of boxes for a few steps with per-instance CFL dt and gather the final
states; rank 0 compares them bit for bit with the whole draw run in one
process. The CPU case runs the oracle; the GPU case runs the device path
(each rank a batch handle of its share on the one GPU: the ranks' kernels do
not wait on one another).
"""
import hashlib
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

STEPS = 6
FIELDS = ("x", "y", "z", "vx", "vy", "vz", "density", "pressure")


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _draw():
    from ultraballpit_b200 import domain
    return domain.batch_boxes(6, seed=11, dx=0.008, lo=300, hi=3000, dims_range=(0.06, 0.14))


def _digest(p) -> str:
    h = hashlib.sha256()
    for f in FIELDS:
        h.update(np.ascontiguousarray(getattr(p, f), np.float32).tobytes())
    return h.hexdigest()


def _run_oracle(scs, idx) -> dict:
    from oracle import oracle as orc
    out = {}
    for i in idx:
        sc = scs[i]
        k = orc.OracleKernel(*sc.kernel_args(), alpha=sc.alpha, beta=sc.beta, tier=1, threads=1, pow_mode=1)
        for _ in range(STEPS):
            k.step(k.compute_timestep(sc.cfl_number))
        out[i] = _digest(k.particles())
    return out


def _run_device(scs, idx) -> dict:
    from ultraballpit_b200.kernel import CudaBatch
    if not idx:
        return {}
    b = CudaBatch([scs[i] for i in idx], device=0)
    b.step_auto(STEPS, want_dt=True)
    out = {i: _digest(b.instance(q)) for q, i in enumerate(idx)}
    b.close()
    return out


def _rank(rank: int, world: int, port: int, mode: str, q) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from ultraballpit_b200.replicas import Replicas, partition_lpt
    rep = Replicas("gloo", timeout_s=120)
    scs = _draw()
    mine = partition_lpt([len(s.particles) for s in scs], rep.world)[rep.rank]
    local = (_run_oracle if mode == "oracle" else _run_device)(scs, mine)
    gathered = rep.gather(local)
    q.put((rank, mine, gathered))
    rep.close()


def _sharded(mode: str):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=600) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return out


def _check(out, whole):
    (r0, mine0, g0), (r1, mine1, g1) = out
    assert (r0, r1) == (0, 1) and g0 == g1
    assert sorted(mine0 + mine1) == list(range(len(whole))) and mine0 and mine1
    merged = {}
    for part in g0:
        merged.update(part)
    assert merged == whole


def test_two_rank_sharded_oracle_run_equals_one_rank_run():
    scs = _draw()
    whole = _run_oracle(scs, list(range(len(scs))))
    assert len(set(whole.values())) == len(scs)
    _check(_sharded("oracle"), whole)


@pytest.mark.gpu
def test_two_rank_sharded_device_run_equals_one_rank_run():
    scs = _draw()
    whole = _run_device(scs, list(range(len(scs))))
    _check(_sharded("device"), whole)
    # and the device run is the oracle's, instance by instance
    assert whole == _run_oracle(scs, list(range(len(scs))))
