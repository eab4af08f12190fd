"""Build the engine library (nedyson_b200/libnedy_b200.so) with nvcc for sm_100a.

    python -m nedyson_b200.build [--force]

The library is built in-tree so that it travels with the repository; it links
only the CUDA runtime.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libnedy_b200.so")
BUILD = os.path.join(HERE, "_build")

SOURCES = ["gemm_f64.cu", "split_gemm.cu", "sigma_df.cu", "sigma_full.cu", "dyson.cu", "boot.cu", "predictor.cu", "capi.cu", "batch.cu", "matsubara.cu", "noalloc.cu", "host_tables.cpp"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I" + os.path.join(ROOT, "include")]


def _nvcc():
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if p and (os.path.isabs(p) and os.path.exists(p) or not os.path.isabs(p)):
            return p
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "nedy.h"))
    objs = []
    nvcc = _nvcc()
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    for s in srcs:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [nvcc] + GENCODE + NVCC_FLAGS + ["-c", src, "-o", obj]
            if s.endswith(".cpp"):
                cmd = [os.environ.get("CXX_HOST", "g++"), "-O3", "-std=c++17", "-fPIC",
                       "-I/usr/local/cuda/include", "-I" + os.path.join(ROOT, "include"), "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(OUT, objs):
        cmd = [nvcc] + GENCODE + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
