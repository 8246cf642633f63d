"""The Rust FFI crate (rust/kernel-cuda/src/ffi.rs) against include/sph_cuda.h.

No Rust toolchain is installed here, so the crate is checked the way a C
compiler sees the ABI: every ``#[repr(C)]`` struct is re-declared in C from
its Rust field list (repr(C) follows the C layout rules) and its size and
field offsets are compared with the header's struct by gcc; every
``extern "C"`` function must match a header prototype in name, parameter
count, parameter types and return type, and every header function must be
declared in the crate.
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FFI = os.path.join(ROOT, "rust", "kernel-cuda", "src", "ffi.rs")
HEADER = os.path.join(ROOT, "include", "sph_cuda.h")

RUST_SCALARS = {"f32": "float", "f64": "double", "i32": "int", "u32": "uint32_t", "u64": "uint64_t",
                "usize": "size_t", "c_int": "int", "u8": "uint8_t", "c_char": "char", "c_void": "void"}
C_ALIASES = {"int32_t": "int", "unsigned": "uint32_t"}


def rust_source() -> str:
    return re.sub(r"//[^\n]*", "", open(FFI).read())


def header_source() -> str:
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    return re.sub(r"#[^\n]*", "", src)


def rust_structs() -> dict:
    out = {}
    for name, body in re.findall(r"#\[repr\(C\)\]\s*(?:#\[derive\([^\]]*\)\]\s*)?pub struct (\w+)\s*\{(.*?)\}",
                                 rust_source(), flags=re.S):
        fields = re.findall(r"(?:pub\s+)?(\w+)\s*:\s*([^,]+?)\s*,", body + ",")
        if fields and fields[0][0] != "_p":
            out[name] = fields
    return out


def rust_type_to_c(t: str) -> tuple[str, str]:
    """(C declaration prefix, array suffix) of a Rust field type."""
    t = t.strip()
    m = re.fullmatch(r"\[(.+);\s*(\d+)\]", t)
    if m:
        base, _ = rust_type_to_c(m.group(1))
        return base, f"[{m.group(2)}]"
    stars = ""
    const = False
    while True:
        m = re.match(r"\*(const|mut)\s+(.*)", t)
        if not m:
            break
        if m.group(1) == "const" and not stars:
            const = True
        stars += "*"
        t = m.group(2).strip()
    base = RUST_SCALARS.get(t, t)
    return ("const " if const else "") + base + stars, ""


def canon_c(decl: str) -> str:
    """Canonical type of a C parameter declaration ('const float *x' ->
    'const float*'; an array parameter decays to a pointer)."""
    decl = decl.strip()
    if decl == "void":
        return ""
    arr = decl.endswith("]")
    decl = re.sub(r"\[\d*\]$", "", decl).strip()
    m = re.match(r"(.*?)(\w+)$", decl)
    if m and m.group(1).strip():
        decl = m.group(1)
    stars = decl.count("*") + (1 if arr else 0)
    words = decl.replace("*", " ").split()
    const = "const" in words
    base = " ".join(w for w in words if w not in ("const", "struct", "enum"))
    base = C_ALIASES.get(base, base)
    return ("const " if const and stars else "") + base + "*" * stars


def canon_rust(t: str) -> str:
    c, arr = rust_type_to_c(t)
    assert not arr, t
    words = c.replace("*", " ").split()
    stars = c.count("*")
    const = words[0] == "const"
    base = " ".join(w for w in words if w != "const")
    base = C_ALIASES.get(base, base)
    return ("const " if const and stars else "") + base + "*" * stars


def rust_functions() -> dict:
    src = rust_source()
    block = re.search(r'extern "C"\s*\{(.*)\}', src, flags=re.S).group(1)
    out = {}
    for name, params, ret in re.findall(r"pub fn (\w+)\s*\((.*?)\)\s*(?:->\s*([^;]+))?;", block, flags=re.S):
        ps = [p.split(":", 1)[1] for p in re.split(r",\s*", params.strip()) if p.strip()]
        out[name] = ([canon_rust(p) for p in ps], canon_rust(ret) if ret else "void")
    return out


def header_functions() -> dict:
    out = {}
    for ret, name, params in re.findall(r"([\w\s\*]+?)\s*\b(sph_\w+)\s*\(([^)]*)\)\s*;", header_source()):
        ret_stars = ret.count("*")
        words = ret.replace("*", " ").split()
        const = "const" in words
        base = " ".join(w for w in words if w != "const")
        r = ("const " if const and ret_stars else "") + C_ALIASES.get(base, base) + "*" * ret_stars
        ps = [canon_c(p) for p in params.split(",")] if params.strip() not in ("", "void") else []
        out[name] = (ps, r)
    return out


def header_struct_fields(name: str) -> int:
    m = re.search(r"typedef struct " + name + r"\s*\{(.*?)\}\s*" + name + ";", header_source(), flags=re.S)
    assert m, name
    count = 0
    for decl in m.group(1).split(";"):
        if decl.strip():
            count += decl.count(",") + 1
    return count


def test_every_header_function_is_bound_with_the_same_signature():
    rust, hdr = rust_functions(), header_functions()
    assert len(hdr) >= 49
    assert sorted(rust) == sorted(hdr)
    for name, (params, ret) in hdr.items():
        assert rust[name] == (params, ret), (name, rust[name], (params, ret))


def test_repr_c_structs_have_the_header_layout(tmp_path):
    structs = rust_structs()
    assert len(structs) >= 14
    lines = ["#include <stdio.h>", "#include <stddef.h>", "#include <stdint.h>", '#include "sph_cuda.h"']
    for name, fields in structs.items():
        lines.append(f"typedef struct RS_{name} {{")
        for fname, ftype in fields:
            decl, arr = rust_type_to_c(ftype)
            lines.append(f"  {decl} {fname}{arr};")
        lines.append(f"}} RS_{name};")
    lines.append("int main(void) {")
    for name, fields in structs.items():
        lines.append(f'printf("{name} %zu %zu\\n", sizeof({name}), sizeof(RS_{name}));')
        for fname, _ in fields:
            lines.append(f'printf("{name}.{fname} %zu %zu\\n", offsetof({name}, {fname}), '
                         f"offsetof(RS_{name}, {fname}));")
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    rows = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines()
    assert rows
    for row in rows:
        key, a, b = row.split()
        assert a == b, key
    for name, fields in structs.items():
        assert header_struct_fields(name) == len(fields), name


def test_abi_constants_match_the_header():
    hdr = open(HEADER).read()
    rs = rust_source()
    for const in ("SPH_OK", "SPH_ERR_INVALID_ARG", "SPH_ERR_OOM", "SPH_ERR_CUDA", "SPH_ERR_NONFINITE",
                  "SPH_ERR_TIMEOUT", "SPH_ERR_CAPACITY", "SPH_ERR_NO_DEVICE", "SPH_ERR_NO_CHECKPOINT",
                  "SPH_BOUNDARY_PARTICLES", "SPH_BOUNDARY_SDF", "SPH_CELL_ORDER_MORTON", "SPH_CELL_ORDER_LINEAR",
                  "SPH_CELL_ORDER_ROWS"):
        want = int(re.search(const + r"\s*=\s*(\d+)", hdr).group(1))
        got = int(re.search(r"pub const " + const + r":\s*\w+\s*=\s*(\d+);", rs).group(1))
        assert got == want, const
    assert re.search(r"#define SPH_MLP_PARAMS (\d+)", hdr).group(1) == \
        re.search(r"pub const SPH_MLP_PARAMS: usize = (\d+);", rs).group(1)
    assert re.search(r"#define SPH_ABI_VERSION (\d+)", hdr).group(1) == \
        re.search(r"pub const SPH_ABI_VERSION: c_int = (\d+);", rs).group(1)


@pytest.mark.parametrize("t,c", [("*const f32", "const float*"), ("*mut *mut SphHandle", "SphHandle**"),
                                 ("c_int", "int"), ("usize", "size_t"), ("*mut c_void", "void*")])
def test_type_mapping(t, c):
    assert canon_rust(t) == c
