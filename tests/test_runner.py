"""The orchestrator's optimistic time stepping (orchestrator runner.rs:189-240).

CPU: the restatement's control flow on a scripted kernel (cooldown, counts,
the dt sequence). GPU: ``CudaKernel.run_optimistic`` (one graph launch a
step, a conditional node for the retry) against the same loop run on the
host through the trait entry points, and against the oracle kernel; states
bit for bit, counters equal."""
import numpy as np
import pytest

from oracle import runner
from oracle.oracle import ErrorMetrics


class ScriptedKernel:
    """Trait stand-in whose density variation after each step() comes from
    a script; records the calls."""

    def __init__(self, variations):
        self.variations = list(variations)
        self.calls = []

    def step(self, dt):
        self.calls.append(("step", dt))

    def save_checkpoint(self):
        self.calls.append(("save",))
        return True

    def restore_checkpoint(self):
        self.calls.append(("restore",))
        return True

    def error_metrics(self):
        return ErrorMetrics(self.variations.pop(0), 0.0, 0.0)


def test_restatement_control_flow():
    k = ScriptedKernel([0.01, 0.05, 0.02, 0.04, 0.0])
    trace = []
    s = runner.run_optimistic(k, 7, lambda: 1e-4, density_limit=0.03, cooldown_steps=2, trace=trace)
    f = np.float32
    safe, opt = float(f(1e-4)), float(f(f(1e-4) * f(1.5)))
    # accept, reject + 2 cooldown steps, accept, reject + ... (the 7th step is a cooldown)
    assert [t[1] for t in trace] == [False, True, False, False, False, True, False]
    assert [t[0] for t in trace] == [opt, safe, safe, safe, opt, safe, safe]
    assert (s.steps, s.accepted, s.rejected, s.cooldown) == (7, 2, 2, 1)
    assert s.sim_time == sum(t[0] for t in trace)
    assert k.calls[:6] == [("save",), ("step", opt), ("save",), ("step", opt), ("restore",), ("step", safe)]
    assert len(k.variations) == 1      # error_metrics only after optimistic steps


def test_kernel_without_checkpoints_steps_safe():
    class NoCk(ScriptedKernel):
        def save_checkpoint(self):
            return False
    k = NoCk([])
    s = runner.run_optimistic(k, 3, lambda: 2e-4)
    assert (s.steps, s.accepted, s.rejected) == (3, 0, 0)
    assert k.calls == [("step", float(np.float32(2e-4)))] * 3


def _dam_break(seed):
    from ultraballpit_b200 import domain
    return domain.dam_break(0.004, seed=seed, block=(0.04, 0.04, 0.04), domain_max=(0.08, 0.04, 0.04),
                            with_sdf=False)


def _mixed_limit(sc, steps, cool):
    """A density-variation limit under which the host loop over this run
    both accepts and rejects optimistic steps: tried among the quantiles of
    the variations a pilot of optimistic steps reaches."""
    from ultraballpit_b200.kernel import CudaKernel
    k = CudaKernel(*sc.kernel_args(), alpha=sc.alpha)
    v = []
    for _ in range(steps):
        k.step(float(np.float32(k.compute_timestep()) * np.float32(1.5)))
        v.append(k.error_metrics().max_density_variation)
    k.close()
    for q in (0.5, 0.75, 0.9, 0.97, 0.25, 0.1):
        limit = float(np.quantile(v, q))
        t = CudaKernel(*sc.kernel_args(), alpha=sc.alpha)
        s = runner.run_optimistic(t, steps, t.compute_timestep, 1.5, limit, cool)
        t.close()
        if s.accepted > 0 and s.rejected > 0:
            return limit
    raise AssertionError(f"no limit splits the run: variations {sorted(v)}")


def _same(a, b):
    for f in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "density", "pressure"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f), err_msg=f)


@pytest.mark.gpu
def test_device_runner_matches_host_loop():
    from ultraballpit_b200.kernel import CudaKernel
    sc = _dam_break(11)
    steps, cool = 30, 2
    limit = _mixed_limit(sc, steps, cool)
    dev = CudaKernel(*sc.kernel_args(), alpha=sc.alpha)
    host = CudaKernel(*sc.kernel_args(), alpha=sc.alpha)
    got = dev.run_optimistic(12, 1.5, limit, cool)
    got = dev.run_optimistic(steps - 12, 1.5, limit, cool)     # counters carry over calls
    want = runner.run_optimistic(host, steps, host.compute_timestep, 1.5, limit, cool)
    assert want.accepted > 0 and want.rejected > 0, (want, limit)
    for key in ("steps", "accepted", "rejected", "cooldown"):
        assert got[key] == getattr(want, key), key
    assert got["sim_time"] == want.sim_time and got["last_dt"] == want.last_dt
    _same(dev.particles(), host.particles())
    dev.close()
    host.close()


@pytest.mark.gpu
def test_device_runner_matches_oracle():
    from oracle import oracle as orc
    from ultraballpit_b200.kernel import CudaKernel
    sc = _dam_break(12)
    steps, cool = 16, 1
    limit = _mixed_limit(sc, steps, cool)
    dev = CudaKernel(*sc.kernel_args(), alpha=sc.alpha, beta=sc.beta)
    cpu = orc.OracleKernel(*sc.kernel_args(), alpha=sc.alpha, beta=sc.beta, tier=1, threads=8, pow_mode=1)
    got = dev.run_optimistic(steps, 1.5, limit, cool)
    want = runner.run_optimistic(cpu, steps, lambda: cpu.compute_timestep(sc.cfl_number), 1.5, limit, cool)
    assert want.rejected > 0, (want, limit)
    assert (got["steps"], got["accepted"], got["rejected"]) == (want.steps, want.accepted, want.rejected)
    assert got["sim_time"] == want.sim_time
    _same(dev.particles(), cpu.particles())
    dev.close()


@pytest.mark.gpu
def test_device_runner_after_caller_steps_and_restore():
    """A caller's own steps, checkpoint restores and changed runner constants
    between runner calls: the runner takes the state as it finds it."""
    from ultraballpit_b200.kernel import CudaKernel
    sc = _dam_break(13)
    a = CudaKernel(*sc.kernel_args(), alpha=sc.alpha)
    b = CudaKernel(*sc.kernel_args(), alpha=sc.alpha)
    sa = a.run_optimistic(5, 1.5, 1.0, 3)
    sb = runner.run_optimistic(b, 5, b.compute_timestep, 1.5, 1.0, 3)
    for k in (a, b):
        k.save_checkpoint()
        k.step(1e-4)
        assert k.restore_checkpoint()
    sa = a.run_optimistic(6, 1.25, 0.0, 2)            # every optimistic step rejected
    sb = runner.run_optimistic(b, 6, b.compute_timestep, 1.25, 0.0, 2, stats=sb)
    assert (sa["steps"], sa["accepted"], sa["rejected"], sa["cooldown"]) == (11, 5, 2, 0)
    assert (sb.steps, sb.accepted, sb.rejected, sb.cooldown) == (11, 5, 2, 0)
    assert sa["sim_time"] == sb.sim_time
    _same(a.particles(), b.particles())
    a.close()
    b.close()
