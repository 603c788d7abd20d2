"""Build the in-tree native libraries.

  libchidg_gpu.so    CUDA kernels + C ABI (include/chidg_gpu.h), sm_100a only
  libchidg_synth.so  host-only synthetic input generator

Run: python -m chidg_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["chidg_gpu.cu", "fgmres.cu", "batch.cu", "noalloc.cu", "matrix_io.cu", "serve.cu", "euler.cu"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False) -> None:
    gpu = os.path.join(HERE, "libchidg_gpu.so")
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "chidg_gpu.h")]
    if force or _stale(gpu, deps):
        _run([NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
              "-o", gpu, *[os.path.join(CSRC, f) for f in CU_SOURCES]])
    synth = os.path.join(HERE, "libchidg_synth.so")
    src = os.path.join(CSRC, "synth.cpp")
    if force or _stale(synth, [src]):
        _run(["g++", "-O3", "-march=x86-64-v3", "-std=c++17", "-fPIC", "-shared", "-pthread", "-o", synth, src])


if __name__ == "__main__":
    build(force="--force" in sys.argv)
