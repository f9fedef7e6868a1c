"""Build libabd_b200.so: hand-written sm_100a CUDA behind the C ABI of include/abd_b200.h.

Compiled in-tree with nvcc (``-gencode arch=compute_100a,code=sm_100a``) so the shared
library sits next to the package and is the one the Python layer loads.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libabd_b200.so")
SOURCES = ["lbvh.cu", "broad.cu", "narrow.cu", "linesearch.cu", "solver.cu", "newton.cu", "sim.cu", "noalloc.cu", "peak.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build(verbose: bool = False, extra=()) -> str:
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    from concurrent.futures import ThreadPoolExecutor

    objs, cmds = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmds.append([nvcc(), *ARCH, *FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
        if verbose:
            print(" ".join(cmds[-1]), file=sys.stderr)
    # the translation units compile independently: one nvcc per unit, in parallel
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        for f in [ex.submit(subprocess.check_call, c) for c in cmds]:
            f.result()
    cmd = [nvcc(), *ARCH, "-shared", "-o", OUT, *objs, "-lcudart"]
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(verbose=True, extra=sys.argv[1:]))
