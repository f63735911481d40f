"""Build the b200tau shared library (sm_100a) in-tree: lsms_b200/_lib/libb200tau.so.

    python -m lsms_b200.build
"""

from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libb200tau.so")
SOURCES = ["capi.cu", "kkr_build.cu", "block_lu.cu", "tc_update.cu", "sweep.cu", "sweep_flow.cu", "adjoint.cu", "noalloc.cu", "angular.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, "common.cuh"), os.path.join(CSRC, "cplx.cuh"), os.path.join(CSRC, "gj.cuh"),
                   os.path.join(CSRC, "cluster.cuh"), os.path.join(CSRC, "umma.cuh"),
                   os.path.join(HERE, "..", "include", "b200tau.h")]
    if (not force and os.path.exists(LIB_PATH)
            and all(os.path.getmtime(LIB_PATH) >= os.path.getmtime(d) for d in deps)):
        return LIB_PATH
    cmd = [nvcc(), "-shared", "-Xcompiler", "-fPIC", "-O3", "-lineinfo", "-std=c++17", *ARCH,
           "-o", LIB_PATH, *srcs]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stderr[-4000:])
    if verbose:
        print(res.stderr)
    return LIB_PATH


if __name__ == "__main__":
    print(build(verbose=True, force=True))
