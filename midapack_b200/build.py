"""Builds libmidapack_b200.so in-tree with nvcc for sm_100a.

    python -m midapack_b200.build      (or __graft_entry__.build())
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmidapack_b200.so")
SOURCES = ["pointing.cu", "toeplitz.cu", "ninv4.cu", "solver.cu", "twolevel.cu", "ecg.cu", "multirhs.cu", "noise.cu", "templates.cu",
           "dropin.cu"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    common = [
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
        "-I", os.path.join(ROOT, "include"), "-I", CSRC,
    ] + (extra or [])
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [nvcc(), "-c", os.path.join(CSRC, src), "-o", obj] + common
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    link = [nvcc(), "-shared", "-o", LIB] + objs + [
        "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "shared",
        "-Xlinker", "-rpath,/usr/local/cuda/lib64"]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.run(link, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
