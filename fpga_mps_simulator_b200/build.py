"""Build libmpsb200.so in-tree with nvcc for sm_100a.

    python -m fpga_mps_simulator_b200.build [--verbose-ptxas]

Each .cu file under csrc/ is compiled to an object (skipped when the object
is newer than its sources and headers), then linked into
fpga_mps_simulator_b200/libmpsb200.so.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmpsb200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: set NVCC or put CUDA 12.9 on PATH")


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def build(verbose_ptxas: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj)
                and os.path.getmtime(obj) >= _newest([src] + headers)):
            continue
        cmd = [nvcc, *ARCH, *FLAGS, "-rdc=false", "-c", src, "-o", obj]
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        subprocess.run([nvcc, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", LIB, *objs,
                        "-lcudart", "-Xlinker", "-z,defs"], check=True)
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="--verbose-ptxas" in sys.argv, force="--force" in sys.argv)
    print(LIB)
