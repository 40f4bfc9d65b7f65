"""Build the engine's shared libraries in-tree.

``build_cuda()`` compiles the product library ``profess_b200/_lib/libprofess_b200.so``
for sm_100a with nvcc.  ``build_emu()`` compiles the same block functions for
the host into ``tests/_emu/libprofess_b200_emu.so``, a test harness that runs
each CUDA block with one thread so the CPU test suite can check the kernels'
logic against the oracle; the product never loads it.

Usage: python -m profess_b200.build [cuda|emu|all]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB_DIR = os.path.join(HERE, "_lib")
EMU_DIR = os.path.join(ROOT, "tests", "_emu")
LIB_PATH = os.path.join(LIB_DIR, "libprofess_b200.so")
EMU_PATH = os.path.join(EMU_DIR, "libprofess_b200_emu.so")

SOURCES = ["engine.cu"]
HEADERS = ["cx.cuh", "fft.cuh", "dcsrch.cuh", "slot.cuh", "ntn_ctl.cuh", "passes.cuh", "setup.cuh", "ewald.cuh", "stress.cuh"]

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fopenmp", "-lgomp",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale(target: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS if os.path.exists(os.path.join(CSRC, f))]
    deps.append(os.path.join(INCLUDE, "profess_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build_cuda(force: bool = False, extra=None) -> str:
    if not force and not _stale(LIB_PATH):
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    cmd = [_nvcc()] + NVCC_FLAGS + (extra or []) + ["-I", INCLUDE, "-I", CSRC]
    cmd += [os.path.join(CSRC, s) for s in SOURCES] + ["-o", LIB_PATH]
    subprocess.run(cmd, check=True)
    return LIB_PATH


def build_emu(force: bool = False) -> str:
    if not force and not _stale(EMU_PATH):
        return EMU_PATH
    os.makedirs(EMU_DIR, exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-DOFDFT_EMU", "-x", "c++",
           "-I", INCLUDE, "-I", CSRC, os.path.join(CSRC, "engine.cu"), "-o", EMU_PATH]
    subprocess.run(cmd, check=True)
    return EMU_PATH


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("cuda", "all"):
        print(build_cuda(force=True))
    if what in ("emu", "all"):
        print(build_emu(force=True))
