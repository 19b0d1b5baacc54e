"""Builds libmkf_b200.so in-tree (mkf_b200/_lib/) with nvcc for sm_100a, and
its debug-build twin libmkf_b200_debug.so (MKF_DEBUG: bounds checks in the
kernels, canary words around every scratch allocation).

    python -m mkf_b200.build [--force] [--debug]
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT, "libmkf_b200.so")
LIB_DEBUG = os.path.join(OUT, "libmkf_b200_debug.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def _deps():
    return glob.glob(os.path.join(SRC, "*.cuh")) + glob.glob(os.path.join(SRC, "*.h")) + \
        [os.path.join(ROOT, "include", "mkf_b200.h")]


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _compile(src, force, debug=False):
    odir = os.path.join(OUT, "debug") if debug else OUT
    obj = os.path.join(odir, os.path.basename(src) + ".o")
    if force or _stale(obj, [src] + _deps()):
        cmd = [NVCC] + ARCH + FLAGS + (["-DMKF_DEBUG"] if debug else []) + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, debug: bool = False) -> str:
    os.makedirs(os.path.join(OUT, "debug") if debug else OUT, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(SRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, debug), srcs))
    lib = LIB_DEBUG if debug else LIB
    if force or _stale(lib, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, debug="--debug" in sys.argv))
