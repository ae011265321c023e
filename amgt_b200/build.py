"""Builds libamgt_b200.so in-tree with nvcc for sm_100a (B200).

python amgt_b200/build.py [-v]   (run as a file: importing the package
                                 loads the library this script builds)
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libamgt_b200.so")
SOURCES = ["runtime.cu", "convert.cu", "spmv.cu", "spgemm.cu", "hypre_mirror.cu", "noalloc.cu", "amg.cu", "packed.cu",
           "spmm_tc.cu", "autotune.cu", "multirhs.cu", "batch.cu", "policy.cu", "boomer.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off", "-cudart", "static",
         "--expt-relaxed-constexpr"]
# host code parallelised with OpenMP (BoomerAMG's coarsening on the host)
OPENMP = {"boomer.cu": ["-Xcompiler", "-fopenmp"]}


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "amgt_b200.h"))
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_info:
            cmd = [NVCC, *ARCH, *FLAGS, *OPENMP.get(src, []), "-c", s, "-o", o]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if _stale(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-Xcompiler", "-fopenmp", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="-v" in sys.argv))
