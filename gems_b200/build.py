"""Build the sm_100a shared library gems_b200/libgemsgpu.so with nvcc.

The library is built in-tree so that it travels with the repository; the
compile flags pin the B200 target (compute_100a / sm_100a).
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRCS = [os.path.join(HERE, "csrc", f) for f in ("gemsgpu.cu", "noalloc.cu", "peaks.cu")]
OUT = os.path.join(HERE, "libgemsgpu.so")
DEPS = [os.path.join(HERE, "csrc", f) for f in ("gemsgpu.cu", "noalloc.cu", "peaks.cu", "kernels.cuh", "lbfgs.cuh", "neb.cuh",
                                                             "common.cuh")] + [
    os.path.join(os.path.dirname(HERE), "include", "gemsgpu.h")]

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(d) > t for d in DEPS if os.path.exists(d))


def build(force=False, verbose=False, extra=()):
    if not force and not stale():
        return OUT
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-o", OUT, *SRCS]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force=True, verbose=True, extra=sys.argv[1:])
