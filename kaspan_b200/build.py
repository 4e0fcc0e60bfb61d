"""Builds libkspn.so (all CUDA sources in csrc/) for sm_100a, in-tree.

    python -m kaspan_b200.build [--force] [--verbose]

One nvcc invocation: every .cu under csrc/ compiled with
-gencode arch=compute_100a,code=sm_100a and linked into a shared library
next to this file.  Rebuilds only when a source or header is newer than the
library (or with --force).
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libkspn.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++20",
    "-Xcompiler", "-fPIC,-O3",
    "--expt-relaxed-constexpr", "--extended-lambda",
    "-shared", "-cudart", "static",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    if not force and not _stale():
        return LIB
    cmd = [_nvcc(), *NVCC_FLAGS, "-I", INCLUDE, *(extra or []), *sources(), "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


CLI_SRC = os.path.join(HERE, "cli", "kspn_bench.cpp")
CLI = os.path.join(HERE, "kspn_bench")


def build_cli(force: bool = False) -> str:
    """The bench_kaspan-compatible command line (links libkspn.so)."""
    if not force and os.path.exists(CLI) and os.path.getmtime(CLI) > max(os.path.getmtime(CLI_SRC), os.path.getmtime(LIB)):
        return CLI
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++20", "-I", INCLUDE, CLI_SRC, "-o", CLI + ".tmp", "-L", HERE, "-lkspn", "-Xlinker", "-rpath,$ORIGIN", "-cudart", "static"]
    subprocess.run(cmd, check=True)
    os.replace(CLI + ".tmp", CLI)
    return CLI


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None)
    build_cli(force="--force" in sys.argv)
    print(LIB)
    print(CLI)
