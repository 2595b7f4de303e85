"""Builds the native library and the drop-in executable in-tree.

    python -m <package>.build          (or: python build.py)

Outputs (next to this file, in lib/):
    libtdem_b200.so            CUDA kernels for sm_100a + C++ host code behind include/tdem.h
    tdem_calcnonstat3dline     drop-in for the reference's CalcNonstat3DLine executable

Every .cu file is compiled by nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a); .cpp files go through nvcc's host
compiler.  Objects are rebuilt when their source or any header is newer.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
OBJ_DIR = os.path.join(LIB_DIR, "obj")
LIB = os.path.join(LIB_DIR, "libtdem_b200.so")
EXE = os.path.join(LIB_DIR, "tdem_calcnonstat3dline")
INCLUDE = os.path.normpath(os.path.join(HERE, "..", "include"))

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + CSRC, "-I" + INCLUDE]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: install the CUDA toolkit or set NVCC")


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def build(verbose: bool = False) -> str:
    """Compiles what is out of date and returns the library path."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    nvcc = _nvcc()
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    hdr_time = _newest(headers)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    sources = [s for s in sources if os.path.basename(s) != "cli.cpp"]
    objs, cmds = [], []
    for src in sources:
        obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_time):
            continue
        cmds.append([nvcc] + ARCH + COMMON + ["-c", src, "-o", obj])
    # the out-of-date objects compile side by side (one nvcc process each)
    from concurrent.futures import ThreadPoolExecutor

    def compile_one(cmd):
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(compile_one, c) for c in cmds]:
            f.result()
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    cli = os.path.join(CSRC, "cli.cpp")
    if not os.path.exists(EXE) or os.path.getmtime(EXE) < max(os.path.getmtime(LIB), os.path.getmtime(cli)):
        cmd = [nvcc] + ARCH + COMMON + [cli, "-o", EXE, "-L" + LIB_DIR, "-ltdem_b200",
                                       "-Xlinker", "-rpath=$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
