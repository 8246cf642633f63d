"""Replica plumbing of the benchmark: one process per GPU, each rank runs its
own simulations (no exchange on the data path; weak scaling), and whole-job
numbers are taken over ranks: time as the maximum, work as the sum.

Ranks come from the launcher's environment (RANK, WORLD_SIZE, LOCAL_RANK,
MASTER_ADDR, MASTER_PORT). With one rank no process group is created.
"""
from __future__ import annotations

import os
from datetime import timedelta


def partition_lpt(sizes, parts: int) -> list[list[int]]:
    """Greedy bin-packing of independent instances onto ``parts`` GPUs
    (longest processing time first): instances by decreasing size, each to the
    least-loaded GPU so far (ties: lower index). Deterministic, so every rank
    computes the same assignment without communicating. Returns, per part, the
    instance indices in increasing order."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    load = [0] * parts
    out = [[] for _ in range(parts)]
    for i in order:
        p = min(range(parts), key=lambda q: (load[q], q))
        out[p].append(i)
        load[p] += sizes[i]
    return [sorted(o) for o in out]


def env() -> tuple[int, int, int]:
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Replicas:
    """Process group of the replicas (``backend`` "nccl" on GPUs, "gloo"
    on the host), created only when WORLD_SIZE > 1."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 300.0):
        self.rank, self.world, self.local = env()
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            kw = {}
            if backend == "nccl":
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
            self.dist = dist

    def _reduce(self, x: float, op) -> float:
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        return float(x) if self.dist is None else self._reduce(x, self.dist.ReduceOp.MAX)

    def sum(self, x: float) -> float:
        return float(x) if self.dist is None else self._reduce(x, self.dist.ReduceOp.SUM)

    def gather(self, obj) -> list:
        """Every rank's ``obj`` (picklable), in rank order, on every rank (a
        host gather of per-instance statistics at the end of a run)."""
        if self.dist is None:
            return [obj]
        out = [None] * self.world
        self.dist.all_gather_object(out, obj)
        return out

    def whole_job_rate(self, local_particles: int, steps: int, local_ms: float) -> tuple[float, float]:
        """(particle-steps/s of all ranks together, max ms over ranks): the
        particles of every rank advanced ``steps`` steps in the slowest
        rank's time."""
        ms = self.max(local_ms)
        return self.sum(local_particles) * steps / (ms / 1e3), ms

    def close(self) -> None:
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None
