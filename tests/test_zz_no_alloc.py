"""The allocation-free grid build against the handle's grid.

sph_grid_sort_noalloc serves callers that cannot let a library call
cudaMalloc (an engine that owns all device memory through its own pool, or
one whose other streams must not stall on the synchronization an allocation
can cause). Its output must equal, bit for bit, the grid that the regular
entry points build (sph_create with the linear cell order, read back with
sph_read_grid), on two calls in a row that reuse the same static scratch.
"""
import ctypes as C

import numpy as np
import pytest

from ultraballpit_b200 import domain
from ultraballpit_b200.kernel import CELL_ORDER_LINEAR, CudaKernel, load_library

pytestmark = pytest.mark.gpu

SPH_OK, SPH_ERR_CAPACITY = 0, 6
MAX_CELLS = 1 << 19


def _fn():
    L = load_library()
    f = L.sph_grid_sort_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_float),
                  C.POINTER(C.c_float), C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_size_t, C.c_void_p]
    f.restype = C.c_int
    return f


def _f3(v):
    return (C.c_float * 3)(*map(float, v))


def grid_noalloc(x, y, z, sc):
    """Run the entry point on device copies of x, y, z; return host arrays."""
    import torch
    dev = torch.device("cuda", 0)
    n = x.shape[0]
    cell = np.float32(2.0) * np.float32(sc.h)
    dims = [max(int(np.ceil(np.float32(np.float32(sc.domain_max[a]) - np.float32(sc.domain_min[a])) / cell)), 1)
            for a in range(3)]
    ncells = dims[0] * dims[1] * dims[2]
    tx, ty, tz = (torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev) for a in (x, y, z))
    idx = torch.empty(n, dtype=torch.int32, device=dev)
    off = torch.empty(ncells, dtype=torch.int32, device=dev)
    cnt = torch.empty(ncells, dtype=torch.int32, device=dev)
    srt = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = _fn()(tx.data_ptr(), ty.data_ptr(), tz.data_ptr(), n, _f3(sc.domain_min), _f3(sc.domain_max),
               float(cell), idx.data_ptr(), off.data_ptr(), cnt.data_ptr(), srt.data_ptr(), ncells, stream)
    assert st == SPH_OK, st
    return {k: t.cpu().numpy().view(np.uint32) for k, t in
            dict(cell_index=idx, offsets=off, counts=cnt, sorted=srt).items()}


def _assert_grid_equal(a, g):
    np.testing.assert_array_equal(a["cell_index"], g["cell_linear"])
    np.testing.assert_array_equal(a["counts"], g["cell_count"])
    np.testing.assert_array_equal(a["offsets"], g["cell_start"])
    np.testing.assert_array_equal(a["sorted"], g["slot_id"])


def test_noalloc_grid_matches_handle_grid_on_two_calls():
    """Two calls in a row on different grids and sizes share the scratch."""
    sc1 = domain.dam_break(0.004, seed=77, with_sdf=False)
    k1 = CudaKernel(*sc1.kernel_args(), alpha=sc1.alpha, cell_order=CELL_ORDER_LINEAR)
    for _ in range(5):
        k1.step(k1.compute_timestep())
    q = k1.particles()  # positions of the last force computation's grid
    first = grid_noalloc(q.x, q.y, q.z, sc1)
    _assert_grid_equal(first, k1.read_grid())

    sc2 = domain.dam_break(0.002, seed=78, block=(0.06, 0.05, 0.04), domain_max=(0.12, 0.1, 0.08),
                           with_sdf=False)
    k2 = CudaKernel(*sc2.kernel_args(), alpha=sc2.alpha, cell_order=CELL_ORDER_LINEAR)
    p = sc2.particles
    second = grid_noalloc(p.x, p.y, p.z, sc2)
    _assert_grid_equal(second, k2.read_grid())
    assert first["sorted"].shape != second["sorted"].shape
    assert first["counts"].shape != second["counts"].shape


def test_noalloc_rejects_grids_beyond_its_scratch():
    f = _fn()
    # 2h = 1 mm over a 1 m cube: 1e9 cells, far beyond SPH_NOALLOC_MAX_CELLS
    st = f(None, None, None, 0, _f3((0, 0, 0)), _f3((1, 1, 1)), 0.001, None,
           C.c_void_p(1), C.c_void_p(1), None, 10**9, None)
    assert st == SPH_ERR_CAPACITY
