"""Builds the native library in-tree: hpgem_b200/_lib/libhpgem_b200.so.

nvcc compiles the CUDA translation units (csrc/*.cu: the C ABI, the stage
launchers, the batch and serving loop) for sm_100a only, together with the
C++ host set-up (csrc/host/*.cpp), one object per source in parallel
(objects under hpgem_b200/_build/, rebuilt when their source or any header
changed), then links them.  Run ``python -m hpgem_b200.build``.
"""
import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIB_DIR, "libhpgem_b200.so")
SOURCES = sorted(glob.glob(os.path.join(CSRC, "*.cu"))) + [
    os.path.join(CSRC, "host", "setup.cpp"),
    os.path.join(CSRC, "host", "operators.cpp"),
    os.path.join(CSRC, "host", "linear.cpp"),
    os.path.join(CSRC, "host", "sources.cpp")]
HEADERS = sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + sorted(glob.glob(os.path.join(CSRC, "host", "*.h"))) + [
    os.path.join(CSRC, "host", "simplex_rules.inc"),
    os.path.join(os.path.dirname(HERE), "include", "hpgem_b200.h")]
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC"]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _obj(src):
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    return os.path.join(OBJ_DIR, rel + ".o")


def _newest_header():
    return max((os.path.getmtime(p) for p in HEADERS if os.path.exists(p)), default=0.0)


def _stale(src, hdr_time):
    o = _obj(src)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    return os.path.getmtime(src) > t or hdr_time > t


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in SOURCES + HEADERS if os.path.exists(p))


def _compile(src, verbose):
    o = _obj(src)
    tmp = o + ".tmp%d" % os.getpid()
    cmd = [nvcc()] + FLAGS + (["-Xptxas=-v"] if verbose else []) + ["-c", src, "-o", tmp]
    subprocess.run(cmd, check=True)
    os.replace(tmp, o)
    return o


def build(force=False, verbose=False, jobs=None):
    if not force and up_to_date():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    hdr = _newest_header()
    todo = [s for s in SOURCES if force or _stale(s, hdr)]
    with ThreadPoolExecutor(max_workers=jobs or min(len(SOURCES), os.cpu_count() or 4)) as pool:
        list(pool.map(lambda s: _compile(s, verbose), todo))
    tmp = LIB + ".tmp%d" % os.getpid()
    subprocess.run([nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp] +
                   [_obj(s) for s in SOURCES], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
