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
    obj_dir = os.path.join(LIB_DIR, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    common = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O3,-ffp-contract=off",
              "-I", os.path.join(REPO, "include")]
    if ptxas_info:
        common += ["-Xptxas", "-v"]

    def compile_one(f):  # one translation unit (they only share host launch wrappers)
        obj = os.path.join(obj_dir, f + ".o")
        cmd = common + ["-c", os.path.join(CSRC, f), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        return obj, subprocess.run(cmd, capture_output=True, text=True)

    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(len(SOURCES)) as ex:
        done = list(ex.map(compile_one, SOURCES))
    for obj, r in done:
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed ({r.returncode}) on {obj}:\n{r.stdout}\n{r.stderr}")
        if ptxas_info:
            sys.stdout.write(r.stderr)
    cuda_lib = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "lib64")
    cmd = [nvcc, *ARCH, "-shared", "-o", GPU_LIB + ".tmp", *[o for o, _ in done], "-lcublas", "-lcusolver",
           "-Xlinker", f"-rpath,{cuda_lib}"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    os.replace(GPU_LIB + ".tmp", GPU_LIB)
    return GPU_LIB


if __name__ == "__main__":
    print(build_gpu_lib(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv))
