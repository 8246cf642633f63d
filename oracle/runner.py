"""CPU restatement of the orchestrator's optimistic time stepping
(backend/crates/orchestrator/src/runner.rs:189-240), written over the
``SimulationKernel`` trait methods so that it drives any kernel object: the
oracle's, or the CUDA kernel through its public entry points (the host loop
the device runner replaces). Test infrastructure: the checker of
``CudaKernel.run_optimistic``, never a product path.

Per step: dt_safe = compute_timestep (runner.rs:204-209); in a cooldown, one
step of dt_safe and cooldown -= 1 (214-217); otherwise save a checkpoint,
step dt_safe * alpha, and if the maximum density variation then exceeds the
limit restore, step dt_safe, count a rejection and start a cooldown
(218-231), else count an acceptance (232-234). sim_time += dt_used in double
(242), steps += 1.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

ALPHA = 1.5            # runner.rs:189 OPTIMISTIC_ALPHA
DENSITY_VAR_LIMIT = 0.03   # runner.rs:190
COOLDOWN_STEPS = 10    # runner.rs:191


@dataclass
class RunStats:
    sim_time: float = 0.0
    steps: int = 0
    accepted: int = 0
    rejected: int = 0
    last_dt: float = 0.0
    cooldown: int = 0


def run_optimistic(kernel, nsteps: int, timestep, alpha: float = ALPHA, density_limit: float = DENSITY_VAR_LIMIT,
                   cooldown_steps: int = COOLDOWN_STEPS, stats: RunStats | None = None,
                   trace: list | None = None) -> RunStats:
    """``timestep()`` returns dt_safe for the kernel's current state (the
    reference's compute_timestep over particles()). ``trace`` (optional)
    receives (dt_used, rejected) per step."""
    s = stats if stats is not None else RunStats()
    f32 = np.float32
    for _ in range(nsteps):
        dt_safe = f32(timestep())
        rejected = False
        if s.cooldown > 0:
            s.cooldown -= 1
            kernel.step(float(dt_safe))
            used = dt_safe
        elif kernel.save_checkpoint():
            dt_try = f32(dt_safe * f32(alpha))
            kernel.step(float(dt_try))
            if f32(kernel.error_metrics().max_density_variation) > f32(density_limit):
                kernel.restore_checkpoint()
                kernel.step(float(dt_safe))
                used = dt_safe
                s.rejected += 1
                s.cooldown = cooldown_steps
                rejected = True
            else:
                used = dt_try
                s.accepted += 1
        else:
            kernel.step(float(dt_safe))
            used = dt_safe
        s.sim_time += float(used)
        s.steps += 1
        s.last_dt = float(used)
        if trace is not None:
            trace.append((float(used), rejected))
    return s
