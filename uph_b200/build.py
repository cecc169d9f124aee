"""Builds the CUDA library in-tree for sm_100a.

    python -m uph_b200.build          # libuph.so and libuph_sph.so next to this file

libuph.so         the C ABI of include/uph.h (kernels + host code)
libuph_sph.so     derivatives() / SearchNeighbors() with the reference's own
                  signatures (include/uph_system.h), linked against libuph.so
libuph_driver.so  a host caller of derivatives() (include/uph_driver.h)

Objects are rebuilt only when a source or header is newer than the object.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC,
          "-ccbin", "g++"]

# (source, extra flags).  The leapfrog and the wall laws (leapfrog.cuh) are
# compiled without multiply-add contraction so their arithmetic rounds
# exactly like the reference's; the REF pass applies the leapfrog in its
# epilogue, and its own pair arithmetic names every fused multiply-add.
CORE_SOURCES = [
    ("host.cpp", []),
    ("celllist.cu", []),
    ("ref_pass.cu", ["--fmad=false"]),
    ("wcsph_pass.cu", []),
    ("integrate.cu", ["--fmad=false"]),
    ("virtual.cu", ["--fmad=false"]),
    ("sim.cu", []),
    ("search_noalloc.cu", []),
    ("tc_gemm.cu", ["@cutlass"]),
    ("node_chain.cu", ["@cutlass"]),
    ("surrogate.cu", []),
]
DROPIN_SOURCES = [("dropin.cpp", ["-Xcompiler", "-fopenmp"])]

LIB = os.path.join(HERE, "libuph.so")
LIB_SPH = os.path.join(HERE, "libuph_sph.so")
# a host caller of the drop-in (include/uph_driver.h): plain C++, OpenMP, no
# fused multiply-add so its leapfrog rounds as the reference's
DRIVER_SRC = os.path.join(CSRC, "driver.cpp")
LIB_DRIVER = os.path.join(HERE, "libuph_driver.so")
CXX = "g++"  # the system compiler (its OpenMP runtime is the one the oracle builds use)


def _headers():
    out = []
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh")):
                out.append(os.path.join(d, f))
    return out


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def cutlass_include() -> str:
    """CUTLASS / CuTe headers (only the UMMA descriptor types are used): the
    copy vendored by the installed flashinfer or tilelang package."""
    import importlib.util
    for pkg, sub in (("flashinfer", ("data", "cutlass", "include")),
                     ("tilelang", ("3rdparty", "cutlass", "include"))):
        spec = importlib.util.find_spec(pkg)
        if spec and spec.submodule_search_locations:
            path = os.path.join(list(spec.submodule_search_locations)[0], *sub)
            if os.path.exists(os.path.join(path, "cute", "arch", "mma_sm100_desc.hpp")):
                return path
    raise RuntimeError("CUTLASS headers with sm100 UMMA descriptors not found")


def _compile(src, flags, verbose):
    flags = [("-I" + cutlass_include()) if f == "@cutlass" else f for f in flags]
    os.makedirs(BUILD, exist_ok=True)
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src + ".o")
    if _newer(obj, [path] + _headers() + [__file__]):
        _run([NVCC] + ARCH + COMMON + flags + ["-c", path, "-o", obj], verbose)
    return obj


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile both libraries; returns the path of libuph.so."""
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    objs = [_compile(s, f + extra, verbose) for s, f in CORE_SOURCES]
    if _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"], verbose)
    dobjs = [_compile(s, f, verbose) for s, f in DROPIN_SOURCES]
    if _newer(LIB_SPH, dobjs + [LIB]):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB_SPH] + dobjs +
             ["-L" + HERE, "-luph", "-Xlinker", "-rpath,$ORIGIN", "-lcudart", "-lgomp"], verbose)
    if _newer(LIB_DRIVER, [DRIVER_SRC, LIB_SPH] + _headers()):
        cuda = os.path.dirname(os.path.dirname(shutil.which(NVCC) or "/usr/local/cuda/bin/nvcc"))
        _run([CXX, "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-shared", "-I" + INCLUDE,
              "-I" + os.path.join(cuda, "include"), "-o", LIB_DRIVER, DRIVER_SRC, "-L" + HERE, "-luph_sph", "-luph",
              "-L" + os.path.join(cuda, "lib64"), "-lcudart", "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
