"""Build libqb (q_b200/libqb.so) for sm_100a, in tree.

    python -m q_b200.build [--force]

Host sources are compiled by nvcc's host compiler; device code is generated
for sm_100a only (-gencode arch=compute_100a,code=sm_100a).  Object files go to
q_b200/_build/; the library is written next to this file so that it travels
with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libqb.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + os.path.join(REPO, "include"),
          "-I" + CSRC]
SOURCES = ["qfiles.cpp", "setup.cpp", "capi.cpp", "engine.cu", "noalloc.cu", "fep.cu", "mlp.cu"]


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = True) -> str:
    os.makedirs(OUT, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    headers += [os.path.join(REPO, "include", f) for f in os.listdir(os.path.join(REPO, "include"))]
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OUT, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [NVCC, *ARCH, *COMMON, "-c", path, "-o", obj]
            if src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"] if os.environ.get("QB_PTXAS_VERBOSE") else []
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
