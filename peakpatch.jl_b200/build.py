"""Builds libppb.so (the C-ABI library) in-tree with nvcc for sm_100a.

Usage: python peakpatch.jl_b200/build.py [--force] [-j N]
Objects go to peakpatch.jl_b200/_build/, the library to
peakpatch.jl_b200/libppb.so.  Each translation unit is recompiled when it or
any header of csrc/ or include/ is newer than its object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libppb.so")
NVCC = os.environ.get("PPB_NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_LIB = "/usr/local/cuda/lib64"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-ccbin", "/usr/bin/g++"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


# per-file flags: the collapse-table integrations must not contract
# multiplies and adds (bit-exact with the CPU restatement)
FILE_FLAGS = {"k_table.cu": ["-fmad=false"], "k_multires.cu": ["-fmad=false"]}


def _compile(src: str, extra: list[str]) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    cmd = [NVCC] + ARCH + FLAGS + FILE_FLAGS.get(os.path.basename(src), []) + extra + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-x", "cu"] + ARCH + FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int = 8, extra: list[str] | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    extra = extra or []
    hdr_mtime = max(os.path.getmtime(h) for h in _headers())
    todo, objs = [], []
    for src in _sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr_mtime):
            todo.append(src)
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            for o in ex.map(lambda s: _compile(s, extra), todo):
                if verbose:
                    print("compiled", o)
    if force or todo or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-L", CUDA_LIB, "-lcufft",
                                                              "-Xlinker", "-rpath=" + CUDA_LIB, "-ccbin", "/usr/bin/g++"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.j, verbose=a.v))
