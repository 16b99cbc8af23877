"""C-ABI checks that need no GPU: the library builds for sm_100a, loads, exports every
symbol include/jpgpu.h declares, and the ctypes mirror matches the C struct layout."""
import ctypes as C
import os
import re
import subprocess

import pytest

from j_presto_b200 import abi, build, engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "jpgpu.h")


def header_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(jp_[a-z_0-9]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return engine.lib()


def test_exports_every_declared_symbol(lib):
    names = header_functions()
    assert len(names) >= 14
    out = subprocess.run(["nm", "-D", "--defined-only", engine.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (jp_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    assert set(names) == set(engine.EXPORTS)


def test_host_only_entry_points(lib):
    p = abi.JpParams()
    lib.jp_default_params(C.byref(p))
    assert p.precision == abi.JP_PREC_MIXED and p.method == abi.JP_METHOD_CANO
    assert p.dt == 2.0 and p.cutoff == 12.0 and p.update == 10 and p.tempco == 2
    assert p.shake_tol == 1e-6 and p.shake_maxit == 1000 and p.icslop == 3
    assert lib.jp_strerror(0) == b"ok"
    assert b"SHAKE" in lib.jp_strerror(1)
    assert lib.jp_strerror(-100) == b"invalid argument or topology"


def test_struct_layout_matches_c(tmp_path):
    """sizeof/offsetof of jp_system and jp_params from gcc equal the ctypes mirror."""
    src = tmp_path / "lay.c"
    fields_s = [f for f, _ in abi.JpSystem._fields_]
    fields_p = [f for f, _ in abi.JpParams._fields_]
    body = ['#include <stdio.h>', '#include <stddef.h>', '#include "jpgpu.h"', "int main(){"]
    body.append('printf("%zu %zu\\n", sizeof(jp_system), sizeof(jp_params));')
    for f in fields_s:
        body.append(f'printf("%zu\\n", offsetof(jp_system, {f}));')
    for f in fields_p:
        body.append(f'printf("%zu\\n", offsetof(jp_params, {f}));')
    body.append("return 0;}")
    src.write_text("\n".join(body))
    exe = tmp_path / "lay"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                           check=True).stdout.split()]
    assert vals[0] == C.sizeof(abi.JpSystem) and vals[1] == C.sizeof(abi.JpParams)
    off = vals[2:]
    exp = [getattr(abi.JpSystem, f).offset for f in fields_s] + \
          [getattr(abi.JpParams, f).offset for f in fields_p]
    assert off == exp


def test_product_has_no_cpu_fallback():
    """The product package never imports the oracle."""
    pkg = os.path.join(ROOT, "j_presto_b200")
    for dp, _, files in os.walk(pkg):
        for f in files:
            if f.endswith(".py"):
                src = open(os.path.join(dp, f)).read()
                assert "import oracle" not in src and "from oracle" not in src
