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
    # an object is rebuilt when its source, a shared header or the flags changed
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    inc = os.path.join(ROOT, "include")
    headers += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    newest_header = max((os.path.getmtime(h) for h in headers), default=0.0)
    flags_file = os.path.join(objdir, "flags.txt")
    flags = " ".join(common)
    same_flags = os.path.exists(flags_file) and open(flags_file).read() == flags
    jobs, objs = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(obj)
        path = os.path.join(CSRC, src)
        if (same_flags and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(path)
                and os.path.getmtime(obj) >= newest_header):
            continue
        jobs.append([nvcc(), "-c", path, "-o", obj] + common)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(run, c) for c in jobs]:
            f.result()
    with open(flags_file, "w") as f:
        f.write(flags)
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
