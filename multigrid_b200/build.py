"""Builds the CUDA extension libpmg_b200.so in-tree for sm_100a.

The library is a plain shared object with a C ABI (include/pmg_b200.h);
nothing in it depends on torch. Invoked by __graft_entry__.build() and
usable directly: python multigrid_b200/build.py [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libpmg_b200.so")

SOURCES = ["pmg_kernels.cu", "pmg_build.cu", "pmg_solver.cu", "pmg_setup.cc",
           "pmg_noalloc.cu", "pmg_runtime.cc", "pmg_setup_gpu.cu",
           "pmg_io.cc", "pmg_apbs.cu"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    # products and sums are rounded separately, as in the reference
    "--fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-pthread",
    "-I", os.path.join(ROOT, "include"),
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"),
                 "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
               if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "pmg_b200.h"))
    objs = []
    jobs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        objs.append(o)
        if force or not _newer(o, [s] + headers):
            jobs.append([nvcc, *NVCC_FLAGS, "-c", s, "-o", o])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    with ThreadPoolExecutor(max_workers=len(jobs) or 1) as ex:
        list(ex.map(run, jobs))
    if force or jobs or not _newer(LIB, objs):
        run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
             "-cudart", "static", "-o", LIB, *objs, "-lpthread"])
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
