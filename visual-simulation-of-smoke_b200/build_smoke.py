"""Builds libsmoke_b200.so in-tree: CUDA kernels with nvcc for sm_100a, host code with g++ -std=c++23.

Usage: python build_smoke.py [--force]. The library lands next to this file so that it travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsmoke_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

CU_SOURCES = ["step_kernels.cu", "pcg.cu", "mgsolve.cu", "noalloc.cu", "unet.cu"]
CPP_SOURCES = ["context.cpp", "learned.cpp"]
CLI = os.path.join(os.path.dirname(os.path.abspath(__file__)), "smoke_b200_benchmark")
HEADERS = ["smoke_device.cuh", "launch.h", "config_check.h", "grid_sync.cuh", "march.cuh", "unet.h", "tcgen05.cuh", "pdl.cuh"]
INCLUDES = [os.path.join(ROOT, "include"), CSRC]

NVCC_FLAGS = [
    "-std=c++20", "-O3", "-lineinfo", "--expt-relaxed-constexpr",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "-Xptxas", "-warn-spills",
]
CXX_FLAGS = ["-std=c++23", "-O2", "-fPIC", "-Wall", "-Wextra", "-fvisibility=hidden"]


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def _run(cmd):
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + proc.stdout)
    return proc.stdout


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every source that changed and links the shared library. Returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    inc = [f"-I{p}" for p in INCLUDES]
    deps = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", h) for h in os.listdir(os.path.join(ROOT, "include"))]
    dep_time = _newest(deps + [os.path.abspath(__file__)])
    objects = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objects.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(dep_time, os.path.getmtime(s)):
            out = _run([NVCC, *NVCC_FLAGS, *inc, "-c", s, "-o", o])
            if verbose and out:
                print(out)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objects.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(dep_time, os.path.getmtime(s)):
            _run(["g++", *CXX_FLAGS, *inc, f"-I{CUDA_HOME}/include", "-c", s, "-o", o])
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objects):
        _run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB, *objects, "-cudart", "static", "-Xlinker", "--no-undefined"])
    # the benchmark CLI (loads the library, or any library exporting the ABI, at run time)
    cli_src = os.path.join(CSRC, "benchmark_cli.cpp")
    if force or not os.path.exists(CLI) or os.path.getmtime(CLI) < max(dep_time, os.path.getmtime(cli_src)):
        _run(["g++", "-std=c++23", "-O2", "-Wall", "-Wextra", *inc, f"-I{CUDA_HOME}/include", cli_src, "-o", CLI, f"-L{CUDA_HOME}/lib64", "-lcudart_static", "-ldl", "-lpthread", "-lrt"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
