"""Build the in-tree CUDA library gsvit_copy_b200/libgsvit_b200.so for sm_100a.

    python -m gsvit_copy_b200.build [--force] [--verbose-ptxas]

nvcc compiles every source of csrc/ with -gencode arch=compute_100a,code=sm_100a
(cross-compiles without a GPU) and links one shared library that exports the
C ABI of include/gsvit_b200.h.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libgsvit_b200.so")
BUILD = os.path.join(HERE, "_build")

SOURCES = ["fdtd_kernels.cu", "fdtd_bulk.cu", "fdtd_adjoint.cu", "fdtd_api.cu", "plan_host.cpp"]
HEADERS = ["fdtd_internal.h", "fdtd_device.cuh", "fdtd_cells.cuh", "fdtd_cpgroup.cuh", "fdtd_kernels.cuh", "fdtd_bulk.cuh",
           "fdtd_adjoint.cuh", "plan_host.h", os.path.join("..", "..", "include", "gsvit_b200.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.normpath(os.path.join(CSRC, h)) for h in HEADERS]
    objs = []
    common = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp", "--expt-relaxed-constexpr"]
    for src in SOURCES:
        sp = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [sp] + hdrs):
            cmd = [nvcc()] + ARCH + common + ["-c", sp, "-o", obj]
            if src.endswith(".cu") and ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
            subprocess.check_call(cmd)
    if force or _stale(OUT, objs):
        tmp = OUT + ".tmp"
        subprocess.check_call([nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lgomp", "-lcudart"])
        os.replace(tmp, OUT)
    return OUT


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force, a.verbose_ptxas))
    return 0


if __name__ == "__main__":
    sys.exit(main())
