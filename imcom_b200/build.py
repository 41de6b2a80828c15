"""Build ``imcom_b200/libimcom_gpu.so`` (sm_100a) in-tree with nvcc.

Every ``csrc/*.cu`` is compiled for ``-gencode arch=compute_100a,code=sm_100a``
and linked with cuFFT (table FFTs) and cuSOLVER (only the comparison-baseline
eigensolver mode); ``csrc/*.cpp`` holds host-only code (FITS files) and is
compiled with the host C++ compiler.  Object files go to ``imcom_b200/_build``.

Usage: ``python -m imcom_b200.build [--force] [-v]``.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "libimcom_gpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
CXX = os.environ.get("CXX", "g++")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC,
          "--expt-relaxed-constexpr"]
HOST_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-I" + INCLUDE, "-I" + CSRC]
# Files whose arithmetic restates the reference operation by operation.
NO_FMA = {"tables.cu"}


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _deps_mtime():
    m = 0.0
    for f in os.listdir(CSRC):
        m = max(m, os.path.getmtime(os.path.join(CSRC, f)))
    m = max(m, os.path.getmtime(os.path.join(INCLUDE, "imcom_gpu.h")))
    m = max(m, os.path.getmtime(__file__))
    return m


def _compile(src, verbose, extra):
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    if src.endswith(".cpp"):
        cmd = [CXX] + HOST_FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
    else:
        flags = list(COMMON) + ARCH + list(extra)
        if src in NO_FMA:
            flags.append("--fmad=false")
        cmd = [NVCC] + flags + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{cmd[0]} failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, flush=True)
    return obj


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= _deps_mtime():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, extra), srcs))
    cmd = [NVCC, "-shared"] + ARCH + ["-o", OUT + ".tmp"] + objs + [
        "-L" + os.path.join(CUDA, "lib64"), "-lcufft", "-lcusolver", "-lcublas", "-lcudart",
        "-Xlinker", "-rpath," + os.path.join(CUDA, "lib64")]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv or bool(extra), extra=extra))
