"""Build the engine's shared library (libjpgpu.so) in-tree with nvcc for sm_100a.

    python -m j_presto_b200.build          # or j_presto_b200.build.build()

Each .cu in csrc/ is compiled separately (-rdc off) and linked into one C-ABI shared
library; no PyTorch or other framework is linked in.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libjpgpu.so")
SOURCES = ["jp_cells.cu", "jp_pair.cu", "jp_bonded.cu", "jp_integrate.cu", "jp_calib.cu", "jp_abi.cu",
           "jp_noalloc.cu", "jp_gefit.cpp", "jp_mlp.cu", "jp_cmm.cu", "jp_hbond.cu",
           "jp_restraint.cu", "jp_minimize.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_v=False, force=False):
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "jpgpu.h"))
    objs = []
    flags = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include"),
             "-I" + CSRC, "-ftz=false", "-prec-div=true", "-prec-sqrt=true"]
    if ptxas_v:
        flags += ["-Xptxas", "-v"]
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ, os.path.splitext(s)[0] + ".o")
        objs.append(obj)
        if force or ptxas_v or _stale(obj, [src] + headers):
            cmd = [nvcc()] + ARCH + flags + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_v="-v" in sys.argv, force="-f" in sys.argv)
