"""Build the in-tree CUDA library libhercules_b200.so for sm_100a with nvcc."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "libhercules_b200.so")
SRCS = [os.path.join(HERE, "csrc", f) for f in ("hc_api.cu", "hc_noalloc.cu")]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# -split-compile: the device code's kernels are optimised by parallel jobs
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr", "-split-compile", str(os.cpu_count() or 4)]


def sources():
    d = os.path.join(HERE, "csrc")
    return [os.path.join(d, f) for f in sorted(os.listdir(d)) if f.endswith((".cu", ".cuh"))] + \
        [os.path.join(HERE, "..", "include", "hercules_b200.h")]


def needs_build() -> bool:
    if not os.path.exists(SO):
        return True
    t = os.path.getmtime(SO)
    return any(os.path.getmtime(s) > t for s in sources())


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    if force or needs_build():
        cmd = [NVCC] + FLAGS + (extra or []) + ["-o", SO] + SRCS
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return SO


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
