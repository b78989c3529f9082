"""Builds, in-tree, the CUDA library libsemigpu_b200.so (nvcc, sm_100a) and on top of it the
C++ host API libsemigpu_host.so plus the `semiGPU` command-line program.

    python -m semigpu_b200.build [--verbose] [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "capi.cu")
OUT = os.path.join(HERE, "libsemigpu_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-Xcompiler", "-fPIC,-O2", "-shared", "--expt-relaxed-constexpr"]


HOST_DIR = os.path.join(HERE, "host")
HOST_LIB = os.path.join(HERE, "libsemigpu_host.so")
CLI = os.path.join(HERE, "semiGPU")
INC = os.path.join(os.path.dirname(HERE), "include")
CXX = os.environ.get("CXX", "g++")


def sources():
    d = os.path.join(HERE, "csrc")
    return [os.path.join(d, f) for f in sorted(os.listdir(d)) if f.endswith((".cu", ".cuh", ".h"))] + [
        os.path.join(os.path.dirname(HERE), "include", "semigpu_b200.h")]


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in sources())


def build_host(verbose: bool = False) -> None:
    """The C++ façade (reference class names) and the CLI, linked to the CUDA library."""
    common = ["-O2", "-std=c++17", "-fPIC", f"-I{INC}", f"-I{HOST_DIR}"]
    lib = [f"-L{HERE}", "-lsemigpu_b200", "-Wl,-rpath,$ORIGIN"]
    cmds = [[CXX, *common, "-shared", os.path.join(HOST_DIR, "semigpu.cpp"), *lib, "-o", HOST_LIB],
            [CXX, *common, os.path.join(HOST_DIR, "semiGPU.cc"), f"-L{HERE}", "-lsemigpu_host",
             *lib, "-o", CLI]]
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)


def host_up_to_date() -> bool:
    srcs = [os.path.join(HOST_DIR, f) for f in os.listdir(HOST_DIR)] + [OUT]
    return all(os.path.exists(p) for p in (HOST_LIB, CLI)) and all(
        os.path.getmtime(s) <= min(os.path.getmtime(HOST_LIB), os.path.getmtime(CLI)) for s in srcs)


def build(verbose: bool = False, force: bool = False) -> str:
    if force or not up_to_date():
        cmd = [NVCC, *FLAGS, SRC, "-o", OUT]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or not host_up_to_date():
        build_host(verbose)
    return OUT


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
