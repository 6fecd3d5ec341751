"""The Rust facade's #[repr(C)] structs (rust/src/ffi.rs) against the C header they mirror.

This image has no Rust toolchain, so the crate is not compiled here.  Instead its struct declarations are
parsed and restated as C structs with the same field types in the same order; a C compiler then lays out
both those and the header's structs, and every field offset and every struct size must agree (a field
missing from the header does not compile).  #[repr(C)] gives a Rust struct exactly the C layout of its
fields in declaration order, so agreement here is agreement of the two ABIs.  The extern block's function
names must all be declared in the header."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FFI = os.path.join(ROOT, "rust", "src", "ffi.rs")

STRUCTS = {"SspCsc": "ssp_csc", "SspCscOut": "ssp_csc_out", "SspParams": "ssp_params", "SspStats": "ssp_stats",
           "SspSolveOpts": "ssp_solve_opts", "SspSolveReport": "ssp_solve_report",
           "SspServerOpts": "ssp_server_opts", "SspRequest": "ssp_request", "SspResult": "ssp_result",
           "SspServerInfo": "ssp_server_info", "SspProbeResult": "ssp_probe_result"}
SCALARS = {"i32": "int32_t", "i64": "int64_t", "u64": "uint64_t", "f64": "double", "usize": "size_t"}


def _rust_structs():
    src = open(FFI).read()
    out = {}
    for name, body in re.findall(r"#\[repr\(C\)\][^{]*?pub struct (\w+) \{(.*?)\n\}", src, re.S):
        fields = re.findall(r"pub (\w+): ([^,\n]+),", body)
        out[name] = fields
    return out


def _c_decl(name, ty):
    ty = ty.strip()
    if ty in SCALARS:
        return f"{SCALARS[ty]} {name};"
    if ty.startswith("*const") or ty.startswith("*mut"):
        return f"const void* {name};"
    m = re.fullmatch(r"\[c_char; (\d+)\]", ty)
    if m:
        return f"char {name}[{m.group(1)}];"
    if ty in STRUCTS:
        return f"{STRUCTS[ty]} {name};"
    raise AssertionError(f"unmapped Rust type {ty!r} of field {name}")


def test_every_header_struct_has_a_rust_mirror():
    assert set(_rust_structs()) == set(STRUCTS)


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_rust_structs_match_the_header(tmp_path):
    rs = _rust_structs()
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "include/specspars.h"']
    for r, c in STRUCTS.items():
        lines.append(f"typedef struct {{ {' '.join(_c_decl(f, t) for f, t in rs[r])} }} rs_{r};")
    lines.append("int main(void) {")
    labels = []
    for r, c in STRUCTS.items():
        lines.append(f'    printf("%zu %zu\\n", sizeof(rs_{r}), sizeof({c}));')
        labels.append(f"sizeof {r}")
        for f, _ in rs[r]:
            lines.append(f'    printf("%zu %zu\\n", offsetof(rs_{r}, {f}), offsetof({c}, {f}));')
            labels.append(f"{r}.{f}")
    lines += ["    return 0;", "}"]
    src, exe = tmp_path / "rs_layout.c", tmp_path / "rs_layout"
    src.write_text("\n".join(lines) + "\n")
    r = subprocess.run(["gcc", "-std=c11", "-I", ROOT, str(src), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines()
    assert len(got) == len(labels)
    bad = [(lab, g) for lab, g in zip(labels, got) if len(set(g.split())) != 1]
    assert bad == []


def test_rust_extern_functions_are_declared_in_the_header():
    src = open(FFI).read()
    block = src[src.index('extern "C" {'):]
    names = re.findall(r"pub fn (ssp_\w+)\(", block)
    header = open(os.path.join(ROOT, "include", "specspars.h")).read()
    declared = set(re.findall(r"\b(ssp_\w+)\(", header))
    assert len(names) > 30
    assert [n for n in names if n not in declared] == []
