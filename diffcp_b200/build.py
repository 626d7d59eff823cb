"""Builds ``libdiffcp_b200.so`` in-tree for sm_100a with nvcc.

    python -m diffcp_b200.build [--verbose]

The library is a plain C-ABI shared object (no torch symbols); the CUDA
runtime is linked statically so the object loads on hosts without a GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIB_DIR, "libdiffcp_b200.so")
SOURCES = ["kernels.cu", "api.cu", "chamfer_static.cu"]
HEADERS = ["cloth_math.cuh", "dcp_internal.cuh", "dcp_launch.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# The substep kernels divide and take square roots with the approximate forms
# (about 2 ulp); the Chamfer kernels, whose minimum and tie-break follow the
# reference's float32 rounding, use explicitly rounded operations throughout.
EXTRA = {"kernels.cu": ["-prec-div=false", "-prec-sqrt=false"]}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "diffcp_b200.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    objs = []
    for src in SOURCES:
        obj = os.path.join(LIB_DIR, src.replace(".cu", ".o"))
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", *EXTRA.get(src, []), "-Xcompiler", "-fPIC", "-c",
               os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, res.stdout, res.stderr))
        if verbose:
            sys.stdout.write(res.stdout + res.stderr)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc link failed:\n%s%s" % (res.stdout, res.stderr))
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True))
