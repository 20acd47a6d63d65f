"""Builds libcanard_b200.so in-tree with nvcc for sm_100a.

Five objects: the FP64 unit (canard.cu) with -fmad=false, so its kernels keep
the reference's rounding order; the FP32 mixed-precision kernels
(kernels_f32.cu) with multiply-add contraction; host set-up code (host.cpp),
the restart files (restart.cpp) and the Tecplot writer (plt.cpp) with
-ffp-contract=off. Objects go to csrc/_build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
OUT = os.path.join(PKG, "libcanard_b200.so")
BUILD = os.path.join(HERE, "_build")
# (source, FMA contraction allowed)
UNITS = [("canard.cu", False), ("kernels_f32.cu", True), ("host.cpp", False), ("restart.cpp", False),
         ("plt.cpp", False)]
DEPS = [u for u, _ in UNITS] + ["kernels.cuh", "kernels_f32.h", "kernels_setup.cuh", "kernels_tm.cuh", "host.h"]


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


def build(force=False, verbose=False, defines=()):
    if not force and not needs_build():
        return OUT
    hostcxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    os.makedirs(BUILD, exist_ok=True)
    common = [nvcc(), "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off", "-ccbin", hostcxx,
              "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-I", os.path.join(ROOT, "include"), "-I", HERE] + ["-D" + d for d in defines]
    if verbose:
        common.insert(1, "-Xptxas=-v")
    objs, procs = [], []
    for src, fma in UNITS:
        obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        cmd = common + ["-fmad=true" if fma else "-fmad=false", "-c", os.path.join(HERE, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append(subprocess.Popen(cmd))
        objs.append(obj)
    for p in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, "nvcc")
    link = [nvcc(), "-shared", "-ccbin", hostcxx, "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT] + objs + ["-lcudart"]
    subprocess.run(link, check=True)
    return OUT


if __name__ == "__main__":
    build(force=True, verbose="-v" in sys.argv)
    print(OUT)
