"""Build the in-tree CUDA library ``tenax_b200/libtenax_b200.so`` for sm_100a.

    python tenax_b200/build.py   # imports nothing from the package

nvcc cross-compiles without a GPU; the resulting shared object travels with
the source tree.  Rebuilds only when a source is newer than the library.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libtenax_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
SOURCES = ["planner.cpp", "kernels.cu", "gemm_f64.cu", "gemm_tc.cu", "heff_fused.cu", "planner_dev.cu", "svd.cu", "capi.cu"]
HEADERS = ["planner.hpp", "common.cuh", "kernels.cuh", "tcgen05.cuh", "planner_dev.hpp", "svd.hpp"]

NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-lineinfo",
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-Xcompiler",
    "-fPIC",
    "-shared",
    "-cudart",
    "static",
]

# cuSOLVER (sector SVDs), linked dynamically from the CUDA toolkit
LIBS = ["-lcusolver"]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(INCLUDE, "tenax_b200.h")]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), *NVCC_FLAGS, f"-I{INCLUDE}", *srcs, "-o", tmp, *LIBS]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
