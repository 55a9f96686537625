"""Builds the native library libsdpa_b200.so in-tree (sdpa_b200/_lib/), and
the sdpa command-line driver (sdpa_b200/_lib/sdpa) linked against it.

nvcc cross-compiles for sm_100a only (no other architectures, no JIT PTX), so
the build runs on machines without a GPU.  Objects are rebuilt when a source
or header is newer than them.

    python -m sdpa_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT, "libsdpa_b200.so")
# The same library with SDPA_INT = int64_t in class SDPA's signatures, for
# callers built against the reference's ILP64 configuration.
LIB_ILP64 = os.path.join(OUT, "libsdpa_b200_ilp64.so")
CLI_SRC = os.path.join(HERE, "cli", "sdpa_main.cpp")
CLI = os.path.join(OUT, "sdpa")  # the drop-in for the reference's sdpa executable
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-I" + CSRC, "-I" + os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
            + glob.glob(os.path.join(ROOT, "include", "*.h")))


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    hdr_time = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    objs = []
    for src in _sources():
        obj = os.path.join(OUT, os.path.basename(src) + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                and os.path.getmtime(obj) >= hdr_time):
            continue
        cmd = [NVCC] + ARCH + CFLAGS + ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [NVCC] + ARCH + CFLAGS + ["-x", "c++", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    # ILP64: sdpa_call.cpp again with SDPA_INT = int64_t, the other objects shared
    call_src = os.path.join(CSRC, "sdpa_call.cpp")
    call64 = os.path.join(OUT, "sdpa_call.ilp64.o")
    if (force or not os.path.exists(call64) or os.path.getmtime(call64) < os.path.getmtime(call_src)
            or os.path.getmtime(call64) < hdr_time):
        cmd = [NVCC] + ARCH + CFLAGS + ["-DSDPA_INT=int64_t", "-x", "c++", "-c", call_src, "-o", call64]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    objs64 = [o for o in objs if not o.endswith("sdpa_call.cpp.o")] + [call64]
    if force or not os.path.exists(LIB_ILP64) or os.path.getmtime(LIB_ILP64) < max(os.path.getmtime(o)
                                                                                   for o in objs64):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB_ILP64] + objs64 + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(CLI) or os.path.getmtime(CLI) < max(os.path.getmtime(LIB),
                                                                       os.path.getmtime(CLI_SRC)):
        cmd = [os.environ.get("CXX_HOST", "g++"), "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
               CLI_SRC, "-L" + OUT, "-lsdpa_b200", "-Wl,-rpath,$ORIGIN", "-o", CLI]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
