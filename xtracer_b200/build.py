"""Builds the CUDA library libxtgpu.so for sm_100a in-tree (xtracer_b200/_build/).

    python -m xtracer_b200.build          # or: python xtracer_b200/build.py
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libxtgpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I" + os.path.join(HERE, "..", "include")]
# The image's CXX wrapper cannot link OpenMP; nvcc uses the system g++ as host compiler.
CCBIN = ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(HERE, "..", "include", "*.h")))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _deps())


def _compile(src: str, verbose_regs: bool) -> str:
    obj = os.path.join(OUT, os.path.basename(src) + ".o")
    cmd = [NVCC] + CCBIN + ARCH + FLAGS + (["-Xptxas", "-v"] if verbose_regs else []) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    if verbose_regs:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose_regs: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OUT, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_regs), srcs))
    tmp = LIB + ".tmp"
    cmd = [NVCC] + CCBIN + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", tmp] + objs + ["-lcudart", "-lz"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_regs="-v" in sys.argv))
