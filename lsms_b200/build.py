"""Build the b200tau shared library (sm_100a) in-tree: lsms_b200/_lib/libb200tau.so.

    python -m lsms_b200.build
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libb200tau.so")
SOURCES = ["capi.cu", "kkr_build.cu", "block_lu.cu", "tc_update.cu", "sweep.cu", "sweep_flow.cu", "adjoint.cu",
           "noalloc.cu", "pivot.cu", "runtime.cu", "angular.cpp"]
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
    # one object per source, compiled in parallel, then one link
    obj_dir = os.path.join(LIB_DIR, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    flags = ["-Xcompiler", "-fPIC", "-O3", "-lineinfo", "-std=c++17", *ARCH]
    if verbose:
        flags.insert(0, "-Xptxas=-v")
    objs = [os.path.join(obj_dir, os.path.basename(src) + ".o") for src in srcs]

    def compile_one(k):
        return subprocess.run([nvcc(), "-c", *flags, "-o", objs[k], srcs[k]], capture_output=True, text=True)

    with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 1)) as ex:
        results = list(ex.map(compile_one, range(len(srcs))))
    for src, res in zip(srcs, results):
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n" + res.stderr[-4000:])
        if verbose:
            print(os.path.basename(src), res.stderr)
    res = subprocess.run([nvcc(), "-shared", *ARCH, "-o", LIB_PATH, *objs], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + res.stderr[-4000:])
    return LIB_PATH


if __name__ == "__main__":
    print(build(verbose=True, force=True))
