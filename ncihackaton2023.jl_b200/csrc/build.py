"""Builds libsfb200.so (the CUDA kernels + C ABI) for sm_100a, in-tree.

Usage: python build.py [-j N] [--verbose-ptxas]

Each .cu file is compiled to an object under ../_build/ in parallel, and the
objects are linked into ../libsfb200.so next to the Python host package. A file
is recompiled only when it, or any header in this directory, is newer than its
object.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
REPO = os.path.dirname(PKG)
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libsfb200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
         "-I" + os.path.join(REPO, "include")]


def sources():
    return sorted(f for f in os.listdir(HERE) if f.endswith(".cu"))


def headers_mtime():
    hs = [os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(REPO, "include", "sfb200.h"))
    return max(os.path.getmtime(h) for h in hs if os.path.exists(h))


def compile_one(src, ptxas_verbose=False):
    obj = os.path.join(BUILD, src[:-3] + ".o")
    srcp = os.path.join(HERE, src)
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(srcp), headers_mtime()):
        return obj, None
    cmd = [NVCC] + ARCH + FLAGS + (["-Xptxas", "-v"] if ptxas_verbose else []) + ["-c", srcp, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return None, r.stdout + r.stderr
    return obj, (r.stdout + r.stderr) if ptxas_verbose else None


def build(jobs=None, ptxas_verbose=False, quiet=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: compile_one(s, ptxas_verbose), srcs))
    objs = []
    for src, (obj, log) in zip(srcs, results):
        if obj is None:
            sys.stderr.write(f"nvcc failed for {src}:\n{log}\n")
            raise SystemExit(1)
        if log and not quiet:
            sys.stdout.write(log)
        objs.append(obj)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise SystemExit(1)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(a.j, a.verbose_ptxas))
