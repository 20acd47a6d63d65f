"""Builds libcanard_b200.so in-tree with nvcc for sm_100a.

FP64 kernels are compiled with -fmad=false (no multiply-add contraction) so
they keep the reference's rounding order; host code with -ffp-contract=off.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
OUT = os.path.join(PKG, "libcanard_b200.so")
SOURCES = ["canard.cu", "host.cpp"]
DEPS = SOURCES + ["kernels.cuh", "host.h"]


def nvcc():
    for c in ("/usr/local/cuda/bin/nvcc", "nvcc"):
        if os.path.exists(c) or c == "nvcc":
            return c


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    paths = [os.path.join(HERE, f) for f in DEPS] + [os.path.join(ROOT, "include", "canard_gpu.h")]
    return any(os.path.getmtime(p) > t for p in paths)


def build(force=False, verbose=False):
    if not force and not needs_build():
        return OUT
    hostcxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    cmd = [nvcc(), "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-ffp-contract=off",
           "-ccbin", hostcxx,
           "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-fmad=false",
           "-I", os.path.join(ROOT, "include"), "-I", HERE,
           "-o", OUT] + [os.path.join(HERE, f) for f in SOURCES] + ["-lcudart"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force=True, verbose="-v" in sys.argv)
    print(OUT)
