"""Builds the solve-phase library libs2l_gpu.so in-tree for sm_100a (nvcc cross-compiles on a
host without a GPU).  ``python build.py`` or ``build.build_gpu_lib()``."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB_DIR = os.path.join(HERE, "lib")
GPU_LIB = os.path.join(LIB_DIR, "libs2l_gpu.so")
CSRC = os.path.join(HERE, "csrc")
SOURCES = ["kernels.cu", "refactor.cu", "amg.cu", "capi.cu", "amg_setup.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build_gpu_lib(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(REPO, "include", "s2l_gpu.h"),
                                                              os.path.abspath(__file__)]
    if not force and not ptxas_info and _newer(GPU_LIB, deps):
        return GPU_LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O3,-ffp-contract=off", "-shared",
           "-I", os.path.join(REPO, "include"), "-o", GPU_LIB + ".tmp"]
    if ptxas_info:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, f) for f in SOURCES]
    cmd += ["-lcublas", "-lcusolver", "-Xlinker", "-rpath,/usr/local/cuda/lib64"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    if ptxas_info:
        sys.stdout.write(r.stderr)
    os.replace(GPU_LIB + ".tmp", GPU_LIB)
    return GPU_LIB


if __name__ == "__main__":
    print(build_gpu_lib(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv))
