"""In-tree build of the native parts of culbm_b200.

Outputs (next to the sources, so that they travel with the repository):

* ``culbm_b200/libculbm.so`` — the C ABI of ``include/culbm.h`` and every
  sm_100a kernel (nvcc, ``-gencode arch=compute_100a,code=sm_100a``);
* ``culbm_b200/bin/single_dev_expt_main`` — the drop-in CLI driver, host C++
  over the C ABI.

Run ``python -m culbm_b200.build`` or call :func:`build`.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libculbm.so")
BIN_DIR = os.path.join(PKG, "bin")
CLI = os.path.join(BIN_DIR, "single_dev_expt_main")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "--expt-relaxed-constexpr"]
LIB_SOURCES = ["sim.cu", "tile_runtime.cu", "adjoint.cu", "noalloc.cu", "selector.cu"]


def _nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build culbm_b200")
    return path


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _deps():
    files = []
    for d in (CSRC, INCLUDE):
        for name in os.listdir(d):
            if name.endswith((".cu", ".cuh", ".h", ".hpp", ".cpp")):
                files.append(os.path.join(d, name))
    return files + [os.path.abspath(__file__)]


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> None:
    """Compile libculbm.so and the CLI if any source is newer than them."""
    deps = _deps()
    nvcc = _nvcc()
    srcs = [os.path.join(CSRC, s) for s in LIB_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    if force or ptxas_info or not _newer(LIB, deps):
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-shared", "-I", INCLUDE, "-I", CSRC, "-o", LIB, *srcs]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    os.makedirs(BIN_DIR, exist_ok=True)
    if force or not _newer(CLI, deps + [LIB]):
        cmd = ["g++", "-std=c++17", "-O2", "-I", INCLUDE, os.path.join(CSRC, "single_dev_expt_main.cpp"),
               "-L", PKG, "-lculbm", "-Wl,-rpath,$ORIGIN/..", "-o", CLI]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
