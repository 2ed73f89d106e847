"""Build the CUDA library in-tree: voxarmps_b200/libvoxarmps_b200.so (sm_100a).

The translation units with FP64 stages are compiled with -fmad=false: they
keep the reference's two-rounding a*b+c so that their sums match the
oracle's; their FP32 kernels (the mixed-precision viscous sums and inner
SpMV) ask for fused multiply-adds explicitly.  The learned guess's kernels
(mps_gnn.cu) have no FP64 parity to keep and are compiled with contraction.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libvoxarmps_b200.so")
SOURCES = ["mps_context.cu", "mps_neighbors.cu", "mps_stages.cu", "mps_ppe.cu", "mps_noalloc.cu",
           "mps_gnn.cu"]
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills"]
# translation units whose FP64 sums must round as the reference's do
NO_FMA = {"mps_context.cu", "mps_neighbors.cu", "mps_stages.cu", "mps_ppe.cu", "mps_noalloc.cu"}


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "voxarmps.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    objs = []
    for src in SOURCES:
        obj = os.path.join(CSRC, src.replace(".cu", ".o"))
        fma = ["-fmad=false"] if src in NO_FMA else ["-fmad=true"]
        cmd = [NVCC, *ARCH, *FLAGS, *fma, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
