"""TEST INFRASTRUCTURE -- builds the oracle and the reference library used to pin it.

 - oracle/_build/libsmoke_oracle{32,64}.so: the C restatement (smoke_oracle.c) in FP32 and FP64, gcc + OpenMP,
   no FMA contraction, default x86-64 target so the build runs on any host of the same image;
 - oracle/_ref/libvisual-simulation-of-smoke.so: the reference's own backend-cuda.cu compiled for sm_100a
   straight from its sources (one file plus its header; cuBLAS, cuSPARSE and nvtx3 from the CUDA toolkit),
   without its CMake build. Built only when a reference source tree is named (the `tree` argument, the
   --reference-tree flag or the SMOKE_REFERENCE_TREE environment variable) and present; the built file travels
   with the repository copy to the GPU host, which has no reference tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
REF_LIB = os.path.join(REF_OUT, "libvisual-simulation-of-smoke.so")


def _run(cmd):
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + proc.stdout)


def oracle_path(bits: int) -> str:
    return os.path.join(BUILD, f"libsmoke_oracle{bits}.so")


def build_oracle(force: bool = False) -> None:
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "smoke_oracle.c")
    header = os.path.join(ROOT, "include", "visual-simulation-of-smoke-3d.h")
    newest = max(os.path.getmtime(src), os.path.getmtime(header), os.path.getmtime(__file__))
    for bits, define in ((32, []), (64, ["-DORACLE_DOUBLE"])):
        out = oracle_path(bits)
        if force or not os.path.exists(out) or os.path.getmtime(out) < newest:
            _run(["gcc", "-std=c11", "-O3", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                  "-Wall", "-Wno-unknown-pragmas", *define, f"-I{os.path.join(ROOT, 'include')}", src, "-o", out, "-lm"])


def build_reference(tree: str | None = None, force: bool = False) -> bool:
    """Compiles the reference backend for sm_100a from the source tree `tree` (default: $SMOKE_REFERENCE_TREE) if
    its sources are there. Returns True if the library exists."""
    tree = tree or os.environ.get("SMOKE_REFERENCE_TREE")
    src = os.path.join(tree, "backend-cuda.cu") if tree else ""
    if not src or not os.path.exists(src):
        return os.path.exists(REF_LIB)
    os.makedirs(REF_OUT, exist_ok=True)
    if force or not os.path.exists(REF_LIB) or os.path.getmtime(REF_LIB) < os.path.getmtime(src):
        _run([os.path.join(CUDA_HOME, "bin", "nvcc"), "-std=c++20", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
              "--extended-lambda", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-shared",
              "-DVISUAL_SIMULATION_OF_SMOKE_BUILD_SHARED", f"-I{tree}", src, "-o", REF_LIB,
              "-lcublas", "-lcusparse"])
    return True


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--reference-tree", default=None, help="reference source tree (holds backend-cuda.cu)")
    args = ap.parse_args()
    build_oracle(force=args.force)
    print("reference library:", build_reference(args.reference_tree, force=args.force))
