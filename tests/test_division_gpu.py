"""The density, force and XSPH kernels compute q = r / h with sph::div_h
(the reciprocal RN(1/h) and two FMA residual corrections) instead of a
division per pair. The reference divides (kernel/src/sph.rs:38, 66), so q must
be the correctly rounded quotient: this test compares div_h with CUDA's IEEE
division for every float r from 2^-40 to 4h, for the smoothing lengths of the
test and benchmark workloads and for random ones."""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def divlib(tmp_path_factory):
    out = tmp_path_factory.mktemp("div") / "libdivcheck.so"
    csrc = os.path.join(ROOT, "ultraballpit_b200", "csrc")
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "--fmad=false",
                    "-prec-div=true", "-prec-sqrt=true", "-shared", "-Xcompiler", "-fPIC", "-I",
                    os.path.join(ROOT, "include"), "-I", csrc, "-o", str(out),
                    os.path.join(ROOT, "tests", "cuda", "div_check.cu")], check=True)
    lib = ctypes.CDLL(str(out))
    lib.div_check.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_float,
                              ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_uint32)]
    lib.div_check.restype = ctypes.c_int
    return lib


def smoothing_lengths():
    f32 = np.float32
    fixed = [f32(1.3) * f32(dx) for dx in (0.001, 0.002, 0.004, 0.005, 0.01, 0.02, 0.0005, 0.0001)]
    rng = np.random.default_rng(7)
    rand = [f32(v) for v in np.exp(rng.uniform(np.log(1e-4), np.log(0.1), 24))]
    return [float(h) for h in fixed + rand]


@pytest.mark.gpu
@pytest.mark.parametrize("h", smoothing_lengths())
def test_div_h_equals_ieee_division(divlib, h):
    bad, first = ctypes.c_ulonglong(), ctypes.c_uint32()
    lo, hi = float(np.float32(2.0 ** -40)), float(np.float32(4.0 * h))
    assert divlib.div_check(h, lo, hi, ctypes.byref(bad), ctypes.byref(first)) == 0
    assert bad.value == 0, (h, bad.value, np.array([first.value], np.uint32).view(np.float32)[0])
