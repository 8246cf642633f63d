"""CPU-side checks of the C ABI library: it builds, loads, exports every entry
point that include/sph_cuda.h declares, and fails cleanly without a device."""
import ctypes as C
import os
import re
import subprocess

import pytest

from ultraballpit_b200 import build
from ultraballpit_b200 import kernel as K
from ultraballpit_b200 import domain

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions(name="sph_cuda.h"):
    src = open(os.path.join(ROOT, "include", name)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sph_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return C.CDLL(build.LIB_PATH)


def test_library_exports_every_header_symbol(lib):
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(K.EXPORTS) == names


def test_params_default(lib):
    p = K.default_params()
    assert p.alpha == 1.0 and p.beta == 2.0
    assert p.flags == K.FLAGS_REFERENCE and p.cell_order == K.CELL_ORDER_ROWS
    assert p.boundary_mode == K.BOUNDARY_PARTICLES


def test_struct_layouts_match_header(tmp_path):
    """sizeof/offsetof of every ABI struct as a C compiler sees the header."""
    structs = {"SphParams": K.SphParams, "SphParticlesView": K.SphParticlesView,
               "SphParticlesMut": K.SphParticlesMut, "SphBoundaryView": K.SphBoundaryView,
               "SphSdfView": K.SphSdfView, "SphErrorMetrics": K.SphErrorMetrics,
               "SphStepProfile": K.SphStepProfile, "SphGridInfo": K.SphGridInfo,
               "SphSurfaceForce": K.SphSurfaceForce, "SphBodyForce": K.SphBodyForce, "SphLaunch": K.SphLaunch,
               "SphRunStats": K.SphRunStats, "SphDomainSpec": K.SphDomainSpec, "SphBoundaryMut": K.SphBoundaryMut}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "sph_cuda.h"', "int main(void){"]
    for name, cls in structs.items():
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    lines.append("return 0;}")
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                 check=True).stdout.splitlines())
    for name, cls in structs.items():
        assert int(got[name]) == C.sizeof(cls), name
        for fname, _ in cls._fields_:
            assert int(got[f"{name}.{fname}"]) == getattr(cls, fname).offset, (name, fname)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_create_without_device_fails_loudly(lib):
    sc = domain.two_particles()
    with pytest.raises(K.SphError) as e:
        K.CudaKernel(*sc.kernel_args())
    assert e.value.status == 7  # SPH_ERR_NO_DEVICE


def test_null_arguments_rejected(lib):
    L = K.load_library()
    out = C.c_void_p()
    assert L.sph_create(None, None, None, None, C.byref(out)) == 1
    assert L.sph_step(None, C.c_float(1e-4)) == 1
    assert L.sph_particle_count(None) == 0
    assert L.sph_last_error(None) == b"null handle"
