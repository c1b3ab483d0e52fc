"""Build libdada2_b200.so in-tree (sm_100a, CUDA runtime linked statically).

Usage: python dada2-rs_b200/build.py [--force]
The library lands in dada2-rs_b200/dada2_b200/ so it travels with the tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "dada2_b200", "libdada2_b200.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CUDA_HOME = os.path.dirname(os.path.dirname(os.path.realpath(NVCC)))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

SOURCES_CU = ["dgpu_kernels.cu"]
SOURCES_CPP = ["dgpu_host.cpp", "dgpu_service.cpp", "dgpu_derep.cpp", "dgpu_errfun.cpp", "dgpu_errfun_external.cpp"]
HEADERS = ["dgpu_common.h"]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "dada2_b200.h")]
    objs = []
    for src in SOURCES_CU:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [NVCC, "-std=c++17", *ARCH, "-O3", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC",
                   "-I", CSRC, "-I", INCLUDE, "-c", s, "-o", o]
            if verbose_ptxas:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd)
    for src in SOURCES_CPP:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            _run(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra",
                  "-I", CSRC, "-I", INCLUDE, "-I", os.path.join(CUDA_HOME, "include"), "-c", s, "-o", o])
    if force or _stale(OUT, objs):
        _run([NVCC, "-shared", *ARCH, "-cudart", "static", "-o", OUT, *objs, "-lpthread", "-lz"])
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--ptxas-v" in sys.argv)
