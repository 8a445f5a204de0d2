"""Build recipe of libkira_gpu.so (sm_100a only; nvcc cross-compiles without a GPU).

    python -m kira_ls_aligner_b200.build

The library is built in-tree (kira_ls_aligner_b200/lib/) so it travels with the
source tree; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIB_DIR, "libkira_gpu.so")
SOURCES = ["kernels.cu", "wfa.cu", "prefilter.cu", "api.cu", "noalloc.cu", "server.cpp"]
HEADERS = ["common.cuh", "sieve.cuh", "myers.cuh", "bsw.cuh", "bsw16.cuh", "qgram.cuh", "nmmd.cuh",
           "planes.cuh", "addchain.cuh", "wfa.cuh", "internal.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "kira_gpu.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           *[os.path.join(CSRC, s) for s in SOURCES], "-o", LIB + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
