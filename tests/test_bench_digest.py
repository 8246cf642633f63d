"""bench.py marks the ncu traffic record fresh only when it was captured on
the same kernels: a digest of the kernel sources with comments and
whitespace removed. Rewording a comment or reflowing code keeps it; any
change to the code changes it."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_digest_ignores_comments_and_layout_but_not_code():
    b = _bench()
    files = {f: open(os.path.join(ROOT, f), "rb").read()
             for f in b.KERNEL_SOURCES + ["ultraballpit_b200/csrc/sph_api.cu"]}
    base = b.kernel_sources_digest(lambda f: files[f])
    assert base == b.kernel_sources_digest()
    k = b.KERNEL_SOURCES[0]
    reworded = dict(files)
    reworded[k] = files[k].replace(b"// ", b"//  reworded ", 1).replace(b"\n", b"\n\n", 3) + b"/* note */\n"
    assert b.kernel_sources_digest(lambda f: reworded[f]) == base
    edited = dict(files)
    edited[k] = files[k].replace(b"kNbrCap = 128", b"kNbrCap = 64", 1)
    assert edited[k] != files[k]
    assert b.kernel_sources_digest(lambda f: edited[f]) != base
    shapes = dict(files)
    api = "ultraballpit_b200/csrc/sph_api.cu"
    shapes[api] = files[api].replace(b"bs_density = 128", b"bs_density = 256", 1)
    assert shapes[api] != files[api]
    assert b.kernel_sources_digest(lambda f: shapes[f]) != base
