"""Builds libpgb200.so in the package directory, for sm_100a.

    python -m peregrine_b200.build

nvcc cross-compiles without a GPU.  The library is built in-tree so it
travels with the source to wherever it runs.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SOURCES = [os.path.join(HERE, "csrc", "pgb_host.cu"), os.path.join(HERE, "csrc", "pgb_noalloc.cu")]
HEADERS = [os.path.join(HERE, "csrc", f) for f in ("fused.cuh", "fused2.cuh", "layout.cuh", "physics.cuh", "plain.cuh")] + \
          [os.path.join(ROOT, "include", "pgb200.h")]
TARGET = os.path.join(HERE, "libpgb200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "-shared", f"-I{os.path.join(ROOT, 'include')}"]


def stale():
    if not os.path.exists(TARGET):
        return True
    built = os.path.getmtime(TARGET)
    return any(os.path.getmtime(p) > built for p in SOURCES + HEADERS)


def build(force=False, verbose=False):
    if not force and not stale():
        return TARGET
    cmd = [NVCC, *FLAGS, "-o", TARGET, *SOURCES]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return TARGET


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
