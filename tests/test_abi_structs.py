"""The ctypes mirrors of the C ABI's structs (lpa_b200/__init__.py) match
include/lpa_capi.h field for field: a C program built with gcc from the header
prints every field's offset and every struct's size, and ctypes must agree.
A mismatch would hand the library garbage through every call that takes one."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import pytest

import lpa_b200 as L

ROOT = Path(__file__).resolve().parents[1]

MIRRORS = {
    "lpa_graph_desc": L.GraphDesc,
    "lpa_opts": L.Opts,
    "lpa_info": L.Info,
    "lpa_stats": L.Stats,
    "lpa_tune": L.Tune,
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_struct_layouts_match_header(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "lpa_capi.h"', "int main(void) {"]
    for cname, py in MIRRORS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    c_vals = {}
    for line in out:
        if line:
            parts = line.split()
            c_vals[tuple(parts[:-1])] = int(parts[-1])
    for cname, py in MIRRORS.items():
        assert c_vals[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert c_vals[(cname, fname)] == getattr(py, fname).offset, f"{cname}.{fname}"
