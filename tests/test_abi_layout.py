"""The C ABI header compiles as plain C, and every struct the Python mirror
declares has the C compiler's size and field offsets (catches a field added
on one side only)."""
import ctypes as C
import subprocess
from pathlib import Path

import pytest

import gpu_cc_tb_b200 as g

ROOT = Path(__file__).resolve().parent.parent
HDR = ROOT / "include" / "gcc_engine.h"

STRUCTS = {
    "gcc_table_desc": g.TableDesc, "gcc_run_params": g.RunParams, "gcc_result": g.Result,
    "gcc_sched_params": g.SchedParams, "gcc_sched_batch": g.SchedBatch,
    "gcc_sched_result": g.SchedResult, "gcc_oe_desc": g.OeDesc, "gcc_oe_layout": g.OeLayout,
    "gcc_serve_params": g.ServeParams, "gcc_serve_result": g.ServeResult,
}


def test_header_is_plain_c():
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-x", "c", str(HDR)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_python_structs_match_c_layout(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HDR}"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    r = subprocess.run(["gcc", "-std=c99", str(src), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            a, b, c = ln.split()
            got[(a, b)] = int(c)
    for cname, py in STRUCTS.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
