"""The viewer's Frame message (server ws.rs:233-290): the CPU restatement
against a hand-packed known answer, and the device packing against it."""
import struct

import numpy as np
import pytest

from oracle import frame
from ultraballpit_b200.particles import ParticleArrays


def _particles(density, fluid_type):
    n = len(density)
    p = ParticleArrays.from_positions(np.arange(n) * 0.1, np.arange(n) * 0.2, np.arange(n) * 0.3, 0.001)
    p.density[:] = np.asarray(density, np.float32)
    p.fluid_type[:] = np.asarray(fluid_type, np.uint8)
    p.temperature[:] = np.arange(n, dtype=np.float32) + 20.0
    return p


def test_frame_known_answer():
    p = _particles([1000.0, 1050.7, 1.204, 70000.0, np.nan, -5.0], [0, 0, 1, 0, 0, 0])
    # 6 particles, 3 requested: stride 2, particles 0, 2, 4
    got = frame.build_frame(p, 3, 42, 0.125)
    want = struct.pack("<BQId", 2, 42, 3, 0.125)
    for i, ratio in ((0, 1000), (2, 1000), (4, 0)):
        want += struct.pack("<ffffBHB", float(p.x[i]), float(p.y[i]), float(p.z[i]), float(p.temperature[i]),
                            int(p.fluid_type[i]), ratio, 0)
    assert got == want
    np.testing.assert_array_equal(frame.density_ratio(p.density, p.fluid_type), [1000, 1050, 1000, 65535, 0, 0])
    assert len(frame.build_frame(p, 0, 1, 0.0)) == 21          # nothing requested: header only
    assert struct.unpack("<I", frame.build_frame(p, 100, 1, 0.0)[9:13])[0] == 6   # more than n: all


@pytest.mark.gpu
def test_device_frame_matches_restatement():
    from ultraballpit_b200 import domain
    from ultraballpit_b200.kernel import CudaKernel
    sc = domain.dam_break(0.004, seed=5, block=(0.04, 0.04, 0.04), domain_max=(0.08, 0.04, 0.04), with_sdf=False)
    sc.particles.temperature[:] = np.linspace(15.0, 25.0, len(sc.particles)).astype(np.float32)
    k = CudaKernel(*sc.kernel_args(), alpha=sc.alpha)
    for _ in range(5):
        k.step(k.compute_timestep())
    p = k.particles()
    n = len(p)
    for count in (0, 7, n // 20, n - 1, n, 2 * n):
        assert k.pack_frame(count, 9, 0.0375) == frame.build_frame(p, count, 9, 0.0375), count
    k.close()
