"""Builds the engine's shared libraries in-tree (gpu_cross_b200/lib/).

  libxsec_b200.so   CUDA kernels for sm_100a + the C ABI (include/xsec_b200.h)
  libxsec_host.so   C++ host layer mirroring the reference's classes
                    (include/xsec/*.h) on top of the C ABI
  xsec_cross        the reference's main program on that layer

nvcc cross-compiles for sm_100a without a GPU.  Objects are rebuilt when a
source or header is newer than the library.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(CSRC, "host")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "lib")
LIB_CUDA = os.path.join(LIBDIR, "libxsec_b200.so")
LIB_HOST = os.path.join(LIBDIR, "libxsec_host.so")
CLI = os.path.join(LIBDIR, "xsec_cross")

NVCC = os.environ.get("NVCC", "nvcc")
CXX = os.environ.get("CXX", "g++")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I", INCLUDE, "-I", CSRC]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    headers = (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) +
               glob.glob(os.path.join(INCLUDE, "*.h")))
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        if force or _newer(obj, [src, *headers]):
            _run([NVCC, *GENCODE, *NVCC_FLAGS, "-c", src, "-o", obj], verbose)
        objs.append(obj)
    if force or _newer(LIB_CUDA, objs):
        _run([NVCC, *GENCODE, "-shared", "-o", LIB_CUDA, *objs, "-lcudart"], verbose)

    host_srcs = sorted(p for p in glob.glob(os.path.join(HOST, "*.cpp"))
                       if os.path.basename(p) != "main.cpp")
    if host_srcs:
        host_headers = glob.glob(os.path.join(INCLUDE, "xsec", "*.h")) + headers
        if force or _newer(LIB_HOST, [*host_srcs, *host_headers, LIB_CUDA]):
            _run([CXX, "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", "-I", INCLUDE, "-o",
                  LIB_HOST, *host_srcs, "-L", LIBDIR, "-lxsec_b200", "-Wl,-rpath,$ORIGIN",
                  "-ldl", "-pthread"], verbose)
        main = os.path.join(HOST, "main.cpp")
        if os.path.exists(main) and (force or _newer(CLI, [main, *host_headers, LIB_HOST])):
            _run([CXX, "-O2", "-std=c++17", "-Wall", "-I", INCLUDE, "-o", CLI, main, "-L", LIBDIR,
                  "-lxsec_host", "-lxsec_b200", "-Wl,-rpath,$ORIGIN", "-pthread"], verbose)
    return LIB_CUDA


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
