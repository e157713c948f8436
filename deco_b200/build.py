"""In-tree build of the native libraries.

  libdeco_gen.so   host-only synthetic system generator (g++ -fopenmp)
  libdeco_b200.so  sm_100a CUDA kernels + the C ABI declared in include/deco_b200.h
  deco_cpr_gpu     C++ driver that runs the reference's JSON parameter files on the GPU

The shared objects are written next to this file so that they travel with the
source tree; nothing is installed into site-packages.  Rebuilds are mtime-driven.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
INC = os.path.join(ROOT, "include")
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
BUILD = os.path.join(PKG, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("DECO_CXX", "/usr/bin/g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-ccbin", CXX, "-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fopenmp", "-I", INC, "-I", CSRC] + ARCH

GEN_LIB = os.path.join(PKG, "libdeco_gen.so")
GPU_LIB = os.path.join(PKG, "libdeco_b200.so")
DRIVER = os.path.join(PKG, "deco_cpr_gpu")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_gen(verbose=False) -> str:
    src = os.path.join(CSRC, "gen", "generator.cpp")
    deps = [src, os.path.join(INC, "deco_gen.h")]
    if _newer(GEN_LIB, deps):
        _run([CXX, "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=c++17",
              "-I", INC, src, "-o", GEN_LIB], verbose)
    return GEN_LIB


def _cu_sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _headers():
    return (sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + sorted(glob.glob(os.path.join(CSRC, "*.h")))
            + sorted(glob.glob(os.path.join(INC, "*.h"))))


def build_gpu(verbose=False, jobs=None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = _cu_sources()
    hdrs = _headers()
    objs = []
    todo = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if _newer(o, [s] + hdrs):
            todo.append((s, o))
    if todo:
        from concurrent.futures import ThreadPoolExecutor
        def one(so):
            s, o = so
            _run([NVCC] + NVCC_FLAGS + ["-c", s, "-o", o], verbose)
        with ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
            list(ex.map(one, todo))
    if _newer(GPU_LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", GPU_LIB] + objs + ["-Xcompiler", "-fopenmp", "-lcudart"],
             verbose)
    return GPU_LIB


def build_driver(verbose=False) -> str:
    src = os.path.join(HOST, "cpr_gpu.cpp")
    if not os.path.exists(src):
        return ""
    deps = [src] + sorted(glob.glob(os.path.join(HOST, "*.hpp"))) + _headers() + [GPU_LIB, GEN_LIB]
    if _newer(DRIVER, deps):
        cuda = os.path.dirname(os.path.dirname(NVCC))
        _run([CXX, "-O2", "-std=c++17", "-I", INC, "-I", HOST, "-I", os.path.join(cuda, "include"), src, "-o", DRIVER,
              "-L", PKG, "-ldeco_b200", "-ldeco_gen", "-L", os.path.join(cuda, "lib64"), "-lcudart",
              "-Wl,-rpath,$ORIGIN"], verbose)
    return DRIVER


def build_all(verbose=False):
    build_gen(verbose)
    build_gpu(verbose)
    build_driver(verbose)


if __name__ == "__main__":
    build_all(verbose="-v" in sys.argv)
