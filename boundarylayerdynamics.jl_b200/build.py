"""Builds the in-tree engine library ``lib/libbld.so`` for sm_100a.

The library is the C ABI of include/bld.h (kernels + host schedules in
csrc/).  It links the CUDA runtime statically, so the only run-time
dependency is the NVIDIA driver.
"""

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libbld.so")
SOURCES = [os.path.join(HERE, "csrc", "bld_capi.cu")]
DEPS = SOURCES + sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + [
    os.path.join(REPO, "include", "bld.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in DEPS)


def build(force=False, verbose=False, extra=()):
    if not force and up_to_date():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-shared",
           "-I", os.path.join(REPO, "include"), "-I", os.path.join(HERE, "csrc"),
           "-o", LIB + ".tmp", *SOURCES, "-cudart", "static", *extra]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a.startswith("-X")])
    print(LIB)
