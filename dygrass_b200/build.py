"""Build the in-tree shared libraries of dygrass_b200.

libdygrass.so  -- CUDA kernels (sm_100a) + C ABI (include/dyg.h) + synthetic
                  workload generators (include/dyg_synth.h) + MTX I/O.
The command-line tools incremental_update / decremental_update link it.

Usage: python -m dygrass_b200.build [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libdygrass.so")
BIN_INCR = os.path.join(PKG, "bin", "incremental_update")
BIN_DECR = os.path.join(PKG, "bin", "decremental_update")
BIN_DYN = os.path.join(PKG, "bin", "dynamic_update")

CUDA_SOURCES = ["walk.cu", "graph.cu", "rowops.cu", "pipeline.cu", "capi.cu", "noalloc.cu", "stream.cu", "shard.cu",
                "server.cu"]
HOST_SOURCES = ["synth.cpp", "mtx_io.cpp", "kappa.cpp"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps() -> list[str]:
    out = []
    for name in os.listdir(CSRC):
        if name.endswith((".cu", ".cuh", ".cpp", ".h")):
            out.append(os.path.join(CSRC, name))
    inc = os.path.join(ROOT, "include")
    out += [os.path.join(inc, f) for f in os.listdir(inc)]
    return out


def _run(cmd: list[str]) -> None:
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_library(force: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES + HOST_SOURCES]
    if force or _stale(LIB, _deps()):
        _run([_nvcc(), *NVCC_FLAGS, "-shared", "-o", LIB, *srcs])
    return LIB


def build_tools(force: bool = False) -> None:
    os.makedirs(os.path.dirname(BIN_INCR), exist_ok=True)
    for target, main in ((BIN_INCR, "cli_incremental.cpp"), (BIN_DECR, "cli_decremental.cpp"),
                         (BIN_DYN, "cli_dynamic.cpp")):
        src = os.path.join(CSRC, main)
        if not os.path.exists(src):
            continue
        if force or _stale(target, [src, LIB]):
            _run(["g++", "-O2", "-std=c++17", "-o", target, src,
                  "-I" + os.path.join(ROOT, "include"), "-L" + PKG, "-ldygrass",
                  "-Wl,-rpath,$ORIGIN/..", "-L/usr/local/cuda/lib64", "-lcudart"])


def build(force: bool = False) -> None:
    build_library(force)
    build_tools(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
