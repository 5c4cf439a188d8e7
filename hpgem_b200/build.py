"""Builds the native library in-tree: hpgem_b200/_lib/libhpgem_b200.so.

nvcc compiles the CUDA stage kernels and the C ABI (csrc/capi.cu) for sm_100a
only, together with the C++ host set-up (csrc/host/*.cpp).  Run
``python -m hpgem_b200.build``.
"""
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIB_DIR, "libhpgem_b200.so")
SOURCES = [os.path.join(CSRC, "capi.cu"),
           os.path.join(CSRC, "host", "setup.cpp"),
           os.path.join(CSRC, "host", "operators.cpp"),
           os.path.join(CSRC, "host", "linear.cpp")]
DEPS = SOURCES + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [
                  os.path.join(CSRC, "host", "refshapes.h"),
                  os.path.join(CSRC, "host", "setup.h"),
                  os.path.join(CSRC, "host", "operators.h"),
                  os.path.join(CSRC, "host", "linear.h"),
                  os.path.join(CSRC, "host", "simplex_rules.inc"),
                  os.path.join(os.path.dirname(HERE), "include", "hpgem_b200.h")]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in DEPS if os.path.exists(p))


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    tmp = LIB + ".tmp%d" % os.getpid()
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3",
           "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-o", tmp] + SOURCES
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
