"""Build of libpftcc_b200.so: every CUDA source under csrc/ compiled by nvcc for
sm_100a (one object per source, in parallel) and linked into one shared library in
lib/ (kept in-tree so the built file travels with the source tree)."""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libpftcc_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return sources() + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [
        os.path.join(HERE, "..", "include", "pftcc_b200.h"), os.path.abspath(__file__)]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in _deps() if os.path.exists(d))


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: the CUDA library cannot be built")
    return cand


def build(force: bool = False, verbose: bool = False) -> str:
    """compile each source to an object in parallel (nvcc per translation unit), then link"""
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "_build")
    os.makedirs(objdir, exist_ok=True)
    cc = nvcc()
    srcs = sources()
    objs = [os.path.join(objdir, os.path.basename(s)[:-3] + ".o") for s in srcs]
    # a source is recompiled unless its object is newer than it and every shared header
    shared = max(os.path.getmtime(d) for d in _deps() if os.path.exists(d) and not d.endswith(".cu"))
    cmds = [[cc, *ARCH, *FLAGS[:-1], "-c", "-o", o, s] for s, o in zip(srcs, objs)
            if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), shared)]
    if verbose:
        for c in cmds:
            print(" ".join(c))
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds))
    for c, r in zip(cmds, results):
        if r.returncode != 0:
            raise RuntimeError("nvcc failed: " + " ".join(c) + "\n" + r.stdout + r.stderr)
    tmp = LIB + ".tmp"
    link = [cc, *ARCH, "-shared", "-o", tmp, *objs, "-lcufft"]
    if verbose:
        print(" ".join(link))
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
