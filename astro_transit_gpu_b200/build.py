"""Build the engine's shared library in-tree (sm_100a only).

``python -m astro_transit_gpu_b200.build`` compiles ``csrc/bls_engine.cu`` into
``lib/libastrotransit_b200.so`` with nvcc.  The library has a plain C ABI
(``include/astrotransit_b200.h``) and links the CUDA runtime statically, so
it loads next to PyTorch's own runtime without conflicts.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc", "bls_engine.cu")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libastrotransit_b200.so")
HEADER = os.path.join(ROOT, "include", "astrotransit_b200.h")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    # every intended fused multiply-add is written as fma(); nothing else may be
    # contracted, so the engine's arithmetic matches the CPU oracle bit for bit
    "-fmad=false",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the engine needs the CUDA 12.9 toolchain")
    return cand


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    mt = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > mt for p in (SRC, HEADER))


def build(verbose: bool = False, force: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *NVCC_FLAGS, "-o", tmp, SRC]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force=True))
