"""Builds libsalmon_b200.so (the C ABI of include/salmon_gpu.h) for sm_100a.

    python -m salmon_b200.build          # or salmon_b200.build.build()

nvcc compiles every csrc/*.cu into one shared library next to this file, with
the CUDA runtime linked statically so the library does not depend on which
libcudart another module (e.g. torch) has already loaded.  Rebuilds only when
a source or header is newer than the library.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libsalmon_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-shared", "-cudart", "static",
         "--expt-relaxed-constexpr"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def deps():
    return sources() + sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + [
        os.path.join(ROOT, "include", "salmon_gpu.h")]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in deps())


def build(force: bool = False, verbose: bool = False, extra=()):
    if not force and up_to_date():
        return LIB
    cmd = [nvcc()] + ARCH + FLAGS + list(extra) + ["-I", os.path.join(ROOT, "include"), "-o", LIB + ".tmp"] + sources()
    if verbose:
        print(" ".join(cmd))
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + out.stdout + out.stderr)
    if verbose and (out.stdout or out.stderr):
        print(out.stdout + out.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    force = "--force" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    build(force=force or bool(extra), verbose=True, extra=extra)
    print(LIB)
