"""Builds libsalmon_b200.so (the C ABI of include/salmon_gpu.h) for sm_100a.

    python -m salmon_b200.build          # or salmon_b200.build.build()

nvcc compiles every csrc/*.cu to an object (in parallel, one process per
source) and links them into one shared library next to this file, with the
CUDA runtime linked statically so the library does not depend on which
libcudart another module (e.g. torch) has already loaded.

Staleness is decided by content, not by file times: the SHA-256 of every
source, header and flag is written beside the library
(libsalmon_b200.so.sha256), and the library is rebuilt whenever the digest of
the current sources differs from it.  A copied tree whose time stamps moved
therefore neither skips a needed rebuild nor rebuilds needlessly.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libsalmon_b200.so")
DIGEST = LIB + ".sha256"
OBJDIR = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr"]
LFLAGS = ["-shared", "-cudart", "static"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + [os.path.join(ROOT, "include", "salmon_gpu.h")]


def deps():
    return sources() + headers()


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _file_digest(paths, extra=()):
    h = hashlib.sha256()
    for p in paths:
        h.update(os.path.basename(p).encode())
        with open(p, "rb") as f:
            h.update(f.read())
    for e in extra:
        h.update(str(e).encode())
    return h.hexdigest()


def digest(extra=()):
    """Digest of every source, header and flag the library is built from."""
    return _file_digest(deps(), list(ARCH) + CFLAGS + LFLAGS + list(extra))


def up_to_date(extra=()):
    if not (os.path.exists(LIB) and os.path.exists(DIGEST)):
        return False
    with open(DIGEST) as f:
        return f.read().strip() == digest(extra)


def _compile(src, extra, verbose):
    """One source to an object named by its own content digest (headers included)."""
    d = _file_digest([src] + headers(), list(ARCH) + CFLAGS + list(extra))[:20]
    obj = os.path.join(OBJDIR, f"{os.path.splitext(os.path.basename(src))[0]}.{d}.o")
    if os.path.exists(obj) and not extra:
        return obj, ""
    cmd = [nvcc()] + ARCH + CFLAGS + list(extra) + ["-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("nvcc failed on " + os.path.basename(src) + ":\n" + out.stdout + out.stderr)
    os.replace(obj + ".tmp", obj)
    return obj, out.stdout + out.stderr


def build(force: bool = False, verbose: bool = False, extra=()):
    want = digest(extra)
    if not force and up_to_date(extra):
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda s: _compile(s, extra, verbose), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                print(log)
    cmd = [nvcc()] + ARCH + LFLAGS + ["-o", LIB + ".tmp"] + objs
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + out.stdout + out.stderr)
    os.replace(LIB + ".tmp", LIB)
    with open(DIGEST, "w") as f:
        f.write(want + "\n")
    # objects of sources that no longer exist in this form
    keep = set(objs)
    for o in glob.glob(os.path.join(OBJDIR, "*.o")):
        if o not in keep:
            os.remove(o)
    return LIB


if __name__ == "__main__":
    force = "--force" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    build(force=force or bool(extra), verbose=True, extra=extra)
    print(LIB)
