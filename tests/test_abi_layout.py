"""The ctypes mirrors of the public structs (spec_spars_b200/_lib.py) against the C header they mirror: every
field at the same offset and every struct of the same size, as a C compiler lays out include/specspars.h.
A mismatch would make the Python host read or write the wrong bytes across the ABI."""
import ctypes
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PAIRS = {
    "_Csc": "ssp_csc", "_CscOut": "ssp_csc_out", "_Params": "ssp_params", "_Stats": "ssp_stats",
    "_SolveOpts": "ssp_solve_opts", "_SolveReport": "ssp_solve_report", "_ServerOpts": "ssp_server_opts",
    "_Request": "ssp_request", "_Result": "ssp_result", "_ServerInfo": "ssp_server_info",
    "_ProbeResult": "ssp_probe_result",
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_ctypes_structs_match_the_header(tmp_path):
    import spec_spars_b200._lib as L
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "include/specspars.h"', "int main(void) {"]
    expect = []
    for py, c in PAIRS.items():
        S = getattr(L, py)
        lines.append(f'    printf("%zu\\n", sizeof({c}));')
        expect.append((f"sizeof({c})", ctypes.sizeof(S)))
        for f, _ in S._fields_:
            lines.append(f'    printf("%zu\\n", offsetof({c}, {f}));')
            expect.append((f"{c}.{f}", getattr(S, f).offset))
    lines += ["    return 0;", "}"]
    src, exe = tmp_path / "layout.c", tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c11", "-I", ROOT, str(src), "-o", str(exe)], check=True, capture_output=True)
    got = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert len(got) == len(expect)
    bad = [(what, want, int(g)) for (what, want), g in zip(expect, got) if int(g) != want]
    assert bad == []


def test_status_codes_match_the_header():
    """Every SSP_ERR_* the header defines has the same value and name in the Python host's table."""
    import re

    import spec_spars_b200._lib as L
    txt = open(os.path.join(ROOT, "include", "specspars.h")).read()
    codes = {int(v): name for name, v in re.findall(r"#define (SSP_ERR_\w+) \((-\d+)\)", txt)}
    assert len(codes) >= 8 and codes == L.ERROR_NAMES
    assert re.search(r"#define SSP_OK 0\b", txt) and L.SSP_OK == 0
