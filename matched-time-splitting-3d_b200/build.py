"""Builds the in-tree shared library lib/libmts_b200.so for sm_100a.

    python matched-time-splitting-3d_b200/build.py [--force]

Host code (setup, C ABI) and device code are compiled without floating-point
contraction (-fmad=false for the device, -ffp-contract=off for the host): the
plain FP64 path must round every product and sum on its own, as the reference
CPU build does.  The fast FP64 form (fast.cu), whose results are only required
to match the reference to rounding, and the mixed-precision form (mixed.cu),
held to an accuracy bound, are compiled with fused multiply-adds.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libmts_b200.so")
SOURCES = ["setup.cpp", "setup_gpu.cu", "kernels.cu", "mixed.cu", "fast.cu", "diag.cu", "capi.cu"]
HEADERS = ["setup.h", "device.h", "device_common.cuh"]
OBJ_DIR = os.path.join(HERE, "build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# device code of these sources may contract a*b+c into one fused multiply-add
FMA_SOURCES = {"fast.cu", "mixed.cu"}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libmts_b200.so")


def _inputs():
    files = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    files.append(os.path.join(HERE, "..", "include", "mts.h"))
    files.append(os.path.abspath(__file__))
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    flags = ["-O3", "-std=c++17", *ARCH, "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-O3",
             "-Xptxas", "-O3"]

    def compile_one(src):
        obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
        fl = [("-fmad=true" if f == "-fmad=false" and src in FMA_SOURCES else f) for f in flags]
        cmd = [nvcc(), *fl, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        cp = subprocess.run(cmd, capture_output=True, text=True)
        if cp.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src} ({cp.returncode}):\n{cp.stdout}\n{cp.stderr}")
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        objs = list(pool.map(compile_one, SOURCES))
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    cp = subprocess.run(cmd, capture_output=True, text=True)
    if cp.returncode != 0:
        raise RuntimeError(f"link failed ({cp.returncode}):\n{cp.stdout}\n{cp.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=True))
    sys.exit(0)
