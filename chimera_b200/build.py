"""Build libchimera_b200.so in place with nvcc for sm_100a.

The library is plain CUDA C++ behind the C ABI of include/chimera_b200.h; no
torch types cross it, so it is built with nvcc directly rather than as a
torch extension. `build()` is idempotent: it rebuilds only when a source is
newer than the library.
"""
from __future__ import annotations

import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libchimera_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def sources():
    return sorted(glob.glob(os.path.join(SRC, "*.cu")))


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(SRC, "*.cuh")) + [
        os.path.join(ROOT, "include", "chimera_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for s in sources():
        o = os.path.join(objdir, os.path.basename(s)[:-3] + ".o")
        cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-I", os.path.join(ROOT, "include"), "-c", s,
               "-o", o]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((subprocess.Popen(cmd), s))
        objs.append(o)
    for p, s in procs:
        if p.wait() != 0:
            raise RuntimeError(f"nvcc failed on {s}")
    tmp = LIB + f".{os.getpid()}.tmp"
    subprocess.check_call([nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    import sys
    print(build(force="--force" in sys.argv, verbose=True,
                extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else ()))
