"""Builds the sm_100a extension in-tree: exahype_b200/lib/libexahype_b200.so.

  python -m exahype_b200.build [--verbose]

The library exports the C ABI of include/exahype_b200.h and links the CUDA
runtime statically, so it needs nothing from torch at load time.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "lib", "libexahype_b200.so")
SOURCES = ["csrc/capi.cu"]
HEADERS = ["csrc/common.cuh", "csrc/pde.cuh", "csrc/aderdg.cuh", "csrc/predictor_lines.cuh", "csrc/limiter.cuh", "csrc/batch.cuh",
           "csrc/linear.cuh", "csrc/amr.cuh", "csrc/dg_tables.h", "csrc/tmem.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = SOURCES + HEADERS + [os.path.join("..", "include", "exahype_b200.h")]
    return any(os.path.getmtime(os.path.join(HERE, d)) > t for d in deps)


def build(verbose=False, force=False):
    if not force and not needs_build():
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
           "-shared", "-o", tmp] + [os.path.join(HERE, s) for s in SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
