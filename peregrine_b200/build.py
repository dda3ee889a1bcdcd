"""Builds libpgb200.so in the package directory, for sm_100a.

    python -m peregrine_b200.build [--force]

nvcc cross-compiles without a GPU.  The host unit, the no-allocation unit,
the FP64 rate unit and one per-block unit per species count (plain_tu.cu
with PGB_NS = 1..12)
compile in parallel into objects under _build/, then link into one shared
library.  The library is built in-tree so it travels with the source to
wherever it runs.
"""

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
MAXNS = 12
SOURCES = [os.path.join(CSRC, f) for f in ("pgb_host.cu", "pgb_noalloc.cu", "plain_tu.cu", "fp64_peak.cu", "rategen.cu")]
HEADERS = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cuh", ".h"))] + \
          [os.path.join(ROOT, "include", "pgb200.h")]
TARGET = os.path.join(HERE, "libpgb200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", f"-I{os.path.join(ROOT, 'include')}"]


def units():
    """(source, object, extra flags) of every translation unit."""
    out = [(os.path.join(CSRC, "pgb_host.cu"), os.path.join(OBJ, "pgb_host.o"), []),
           (os.path.join(CSRC, "pgb_noalloc.cu"), os.path.join(OBJ, "pgb_noalloc.o"), []),
           (os.path.join(CSRC, "fp64_peak.cu"), os.path.join(OBJ, "fp64_peak.o"), []),
           (os.path.join(CSRC, "rategen.cu"), os.path.join(OBJ, "rategen.o"), [])]
    for n in range(1, MAXNS + 1):
        out.append((os.path.join(CSRC, "plain_tu.cu"), os.path.join(OBJ, f"plain_ns{n}.o"), [f"-DPGB_NS={n}"]))
    return out


def shared_kernels(objs=None):
    """The library's symbols (namespace pgb) that more than one object
    defines.  Each unit holds its own constant memory (species, mechanism),
    so a template instantiated by two units is two kernels reading different
    constants; the linker keeps a single host launch stub for them, and a
    launch may then run either unit's copy.  Empty when every unit's kernels
    are its own."""
    objs = objs if objs is not None else [o for _, o, _ in units()]
    seen = {}
    for obj in objs:
        r = subprocess.run(["nm", "--defined-only", obj], capture_output=True, text=True, check=True)
        for line in r.stdout.splitlines():
            parts = line.split()
            if len(parts) == 3 and parts[1] in ("W", "T") and parts[2].startswith("_ZN3pgb"):
                seen.setdefault(parts[2], []).append(os.path.basename(obj))
    return sorted(f"{name} ({', '.join(where)})" for name, where in seen.items() if len(where) > 1)


def stale():
    if not os.path.exists(TARGET):
        return True
    built = os.path.getmtime(TARGET)
    return any(os.path.getmtime(p) > built for p in SOURCES + HEADERS)


def build(force=False, verbose=False, jobs=None):
    if not force and not stale():
        return TARGET
    os.makedirs(OBJ, exist_ok=True)

    def compile_one(unit):
        src, obj, extra = unit
        cmd = [NVCC, *FLAGS, *extra, "-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(f"nvcc failed on {os.path.basename(src)} {' '.join(extra)}:\n{r.stderr}")
        return obj

    with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as pool:
        objs = list(pool.map(compile_one, units()))
    shared = shared_kernels(objs)
    if shared:
        raise RuntimeError("kernels defined by more than one unit (the linker would keep one launch stub for "
                           "copies that read different constant memory):\n  " + "\n  ".join(shared[:20]))
    cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", TARGET, *objs, "-ldl"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return TARGET


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
