"""Build libsph_cuda.so (sm_100a) in-tree with nvcc.

The WCSPH kernels are compiled with ``--fmad=false`` and IEEE division and
square root (``-prec-div=true -prec-sqrt=true``, denormals kept): every f32
operation then rounds like the reference CPU kernel's, which rustc never
contracts into FMAs. The host side gets ``-ffp-contract=off`` for the same
reason (its precomputed step constants). The CUDA runtime is linked
statically, so the library has no dependency besides the driver.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libsph_cuda.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["sph_api.cu", "sph_noalloc.cu", "sph_mlp.cu", "sph_domain.cu"]
DEPS = ["sph_api.cu", "sph_kernels.cuh", "sph_noalloc.cu", "sph_mlp.cu", "sph_mlp.cuh", "sph_sdf.cuh",
        "sph_domain.cu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def flags(verbose_ptxas: bool = False) -> list[str]:
    f = ARCH + ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-prec-div=true",
                "-prec-sqrt=true", "-ftz=false", "-shared", "-cudart=static",
                "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
                "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    if verbose_ptxas:
        f += ["-Xptxas", "-v"]
    return f


def _stale() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = [os.path.join(CSRC, d) for d in DEPS] + [os.path.join(ROOT, "include", "sph_cuda.h"),
                                                     os.path.abspath(__file__)]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    """Compile the library if any source is newer than it; return its path."""
    if not force and not _stale():
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc()] + flags(verbose_ptxas) + ["-o", tmp] + [os.path.join(CSRC, s) for s in SOURCES]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    if verbose_ptxas:
        sys.stderr.write(r.stderr)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv))
