"""Build libapcloud_gpu.so (sm_100a) in-tree with nvcc.

    python ap-cloud-cosmology_b200/build.py

The library is written next to this file; it is git-ignored but travels with the
repository snapshot to the GPU host.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libapcloud_gpu.so")
SOURCES = ["capi.cu", "scan_sort.cu", "octree_build.cu", "selection.cu", "gfd.cu", "krylov.cu", "mover.cu",
           "noalloc.cu", "mg.cu", "batch.cu", "adjoint.cu", "warmstart.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    newest = max(os.path.getmtime(p) for p in srcs + [os.path.join(CSRC, "apc_internal.cuh"),
                                                       os.path.join(HERE, "..", "include", "apcloud_gpu.h")])
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= newest and not ptxas_info:
        return LIB
    objs = []
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    for s in srcs:
        o = os.path.join(CSRC, os.path.basename(s)[:-3] + ".o")
        cmd = [nvcc(), *NVCC_FLAGS, "-c", s, "-o", o, "-ccbin", "g++"]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True, env=env)
        objs.append(o)
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs,
           "-ccbin", "g++", "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, env=env)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="-v" in sys.argv))
