"""Builds the B200 rigid-body step library in-tree:

    fyzzxyzzy-sdk_b200/lib/libfyzz_b200.so

CUDA sources are compiled for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``) with ``-fmad=false`` so that every float
expression rounds like the reference's x86-64 SSE arithmetic (no fused
multiply-add contraction).  The host engine is C++23 (g++).  Objects are
rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "lib", "obj")
LIB = os.path.join(HERE, "lib", "libfyzz_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++20", "-O3", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC",
              "-Xptxas", "-warn-spills", f"-I{INCLUDE}"] + ARCH
CXX_FLAGS = ["-std=c++23", "-O2", "-fPIC", "-Wall", "-Wextra", "-ffp-contract=off",
             f"-I{os.path.join(CUDA_HOME, 'include')}", f"-I{INCLUDE}"]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(obj, src, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(verbose: bool = False) -> str:
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    os.makedirs(OBJ, exist_ok=True)
    deps = _headers()
    jobs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        if _stale(obj, src, deps):
            jobs.append([NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj])
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cpp"))):
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        if _stale(obj, src, deps):
            jobs.append([shutil.which("g++") or "g++"] + CXX_FLAGS + ["-c", src, "-o", obj])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for log in ex.map(_run, jobs):
                if verbose and log.strip():
                    print(log, file=sys.stderr)
    objs = sorted(glob.glob(os.path.join(OBJ, "*.o")))
    if jobs or not os.path.exists(LIB):
        _run([NVCC, "-shared", "-o", LIB] + objs + ARCH + ["-cudart", "static", "-lpthread"])
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
