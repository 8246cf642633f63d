"""The density scan and the boundary pressure each have two forms: the
warp-cooperative ones (a warp takes its particles cell by cell and tests
candidates 32 at a time with ballot masks) and the per-particle ones; the
library picks by size (at 2048 fluid and 4096 boundary particles per SM).
The small cases here are forced into each form through SPH_WARP_SCAN_MIN and
SPH_ADAMI_CELLS_MIN, read at handle creation, and must equal the oracle bit
for bit in both: the same neighbour lists in the same order and the same
terms in the same order."""
import os

import numpy as np
import pytest

from oracle import oracle as orc
from ultraballpit_b200 import domain
from ultraballpit_b200.kernel import CELL_ORDER_LINEAR, CELL_ORDER_MORTON, CELL_ORDER_ROWS, CudaKernel

from test_parity_gpu import assert_same, small_dam_break

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["warp", "per_particle"])
def form(request, monkeypatch):
    v = "0" if request.param == "warp" else str(1 << 40)
    monkeypatch.setenv("SPH_WARP_SCAN_MIN", v)
    monkeypatch.setenv("SPH_ADAMI_CELLS_MIN", v)
    return request.param


@pytest.mark.parametrize("order", [CELL_ORDER_ROWS, CELL_ORDER_LINEAR, CELL_ORDER_MORTON])
@pytest.mark.parametrize("make", [small_dam_break, domain.water_box_2mm])
def test_both_forms_bit_exact(form, order, make):
    sc = make()
    args = sc.kernel_args()
    gpu = CudaKernel(*args, alpha=sc.alpha, beta=sc.beta, cell_order=order)
    cpu = orc.OracleKernel(*args, alpha=sc.alpha, beta=sc.beta, tier=1, threads=8, pow_mode=1)
    for _ in range(4):
        dt = cpu.compute_timestep(sc.cfl_number)
        gpu.step(dt)
        cpu.step(dt)
        assert_same(gpu.particles(), cpu.particles())
        np.testing.assert_array_equal(gpu.boundary_pressure(), cpu.boundary_pressure())
    gpu.close()
