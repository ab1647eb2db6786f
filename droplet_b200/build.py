"""Build libdroplet_b200.so (sm_100a) in-tree with nvcc.

The library is plain CUDA C++ behind a C ABI (include/droplet_b200.h); no
PyTorch types cross the boundary.  FMA contraction is off (--fmad=false) so
every f32 expression that feeds an integer decision or an output byte is
evaluated exactly as written; the kernels call dl_fma explicitly where a
fused multiply-add is wanted.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdroplet_b200.so")
SOURCES = ["dl_api.cu", "dl_render.cu", "dl_voxel.cu", "dl_mlp.cu", "dl_sorter.cu", "dl_ply.cu", "dl_query.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "--fmad=false",
              "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-Xcompiler", "-ffp-contract=off"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for f in os.listdir(CSRC):
        if os.path.getmtime(os.path.join(CSRC, f)) > t:
            return True
    hdr = os.path.join(HERE, "..", "include", "droplet_b200.h")
    return os.path.exists(hdr) and os.path.getmtime(hdr) > t


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    srcs = [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), *NVCC_FLAGS, "-shared", "-o", tmp, *srcs, "-cudart=static"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
