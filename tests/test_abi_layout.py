"""The ctypes mirror of include/jpgpu.h (j_presto_b200/abi.py) has the C layout: every field
of every struct at the same offset, every struct the same size, as gcc compiles the header
(no GPU)."""
import ctypes
import os
import shutil
import subprocess

import pytest

from j_presto_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = {
    "jp_system": abi.JpSystem, "jp_params": abi.JpParams, "jp_ge": abi.JpGe,
    "jp_ext_cmm": abi.JpExtCmm, "jp_restraints": abi.JpRestraints,
    "jp_min_params": abi.JpMinParams, "jp_ge_fit_params": abi.JpGeFitParams,
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_struct_layouts_match_the_header(tmp_path):
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "jpgpu.h"', "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            s, f, v = line.split()
            got[(s, f)] = int(v)
    for cname, cls in STRUCTS.items():
        assert got[(cname, "sizeof")] == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)

