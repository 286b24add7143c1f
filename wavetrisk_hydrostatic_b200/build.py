"""In-tree build of the native library (libwtgpu.so, sm_100a) and of the oracle.

``build()`` compiles every CUDA source for sm_100a with nvcc and the host grid
builder with g++, links them into ``wavetrisk_hydrostatic_b200/libwtgpu.so``,
and builds the CPU oracle ``oracle/liboracle.so`` (test infrastructure).
Both compile without a GPU.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libwtgpu.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: no contraction of a*b+c, so every operator result is bit-identical
# to the CPU restatement compiled with -ffp-contract=off.
NVCC_FLAGS = ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]
CXX_FLAGS = ["-O2", "-ffp-contract=off", "-fPIC", "-std=c++17"]

CU_SOURCES = ["wt_api.cu", "wt_elliptic.cu", "wt_noalloc.cu", "wt_wavelet.cu", "wt_barotropic.cu", "wt_trend_ml.cu", "wt_remap.cu"]
CPP_SOURCES = ["grid.cpp", "grid_api.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return r


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _deps():
    out = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".cpp", ".hpp", ".h")):
                out.append(os.path.join(d, f))
    return out


def build_lib(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps = _deps()
    if not force and not _newer(LIB, deps):
        return LIB
    jobs = []
    for src in CU_SOURCES:
        path = os.path.join(CSRC, src)
        if os.path.exists(path):
            jobs.append([NVCC, *ARCH, *NVCC_FLAGS, "-c", path, "-o", os.path.join(BUILD, src + ".o")])
    for src in CPP_SOURCES:
        jobs.append(["g++", *CXX_FLAGS, "-c", os.path.join(CSRC, src), "-o", os.path.join(BUILD, src + ".o")])
    # the translation units are independent: compile them side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as ex:
        list(ex.map(_run, jobs))
    objs = [j[-1] for j in jobs]
    tmp = LIB + ".tmp"
    _run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"])
    shutil.move(tmp, LIB)
    return LIB


def build_oracle(force: bool = False) -> str:
    odir = os.path.join(ROOT, "oracle")
    _run(["make", "-C", odir] + (["-B"] if force else []))
    return os.path.join(odir, "liboracle.so")


def build(force: bool = False) -> None:
    build_lib(force)
    build_oracle(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print("built", LIB)
