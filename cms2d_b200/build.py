"""Builds libcmsgpu.so (the CUDA sm_100a library) in-tree with nvcc.

    python -m cms2d_b200.build          # incremental
    python -m cms2d_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libcmsgpu.so")
OBJDIR = os.path.join(HERE, "_build")

SOURCES = ["cms_order.cpp", "cms_flow_geom.cpp", "cms_flow_wetdry.cpp", "cms_solver.cu", "cms_noalloc.cu"]
HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith((".cuh", ".h")))

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    nvcc = _nvcc()
    os.makedirs(OBJDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "cmsgpu.h"), __file__]
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", INCLUDE, "-ccbin", "/usr/bin/g++"]
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(OBJDIR, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + hdrs):
            cmd = [nvcc] + common + ARCH + ["-lineinfo", "-c", path, "-o", obj]
            if src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"] if verbose else []
            else:
                cmd += ["-x", "c++"]
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        subprocess.run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"], check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
