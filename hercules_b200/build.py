"""Build the in-tree CUDA library libhercules_b200.so for sm_100a with nvcc.

The library is rebuilt only when the sources or the flags change: a SHA-256 of
both is kept beside it (libhercules_b200.so.sha256), so a copy of the tree on
another machine uses the prebuilt library whatever its file times say. The
device code is compiled as one module (no -split-compile): split into parallel
chunks, the same sources gave kernels of different speed depending on how they
fell into the chunks (FP64 momentum RHS 1982 against 2262 us a launch at
512x384x256 from two builds of one tree).
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "libhercules_b200.so")
STAMP = SO + ".sha256"
SRCS = [os.path.join(HERE, "csrc", f) for f in ("hc_api.cu", "hc_noalloc.cu")]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr"]


def sources():
    d = os.path.join(HERE, "csrc")
    return [os.path.join(d, f) for f in sorted(os.listdir(d)) if f.endswith((".cu", ".cuh"))] + \
        [os.path.join(HERE, "..", "include", "hercules_b200.h")]


def digest(extra=None) -> str:
    h = hashlib.sha256()
    h.update(" ".join(FLAGS + (extra or [])).encode())
    for s in sources():
        h.update(os.path.basename(s).encode())
        with open(s, "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def needs_build(extra=None) -> bool:
    if not os.path.exists(SO) or not os.path.exists(STAMP):
        return True
    with open(STAMP) as f:
        return f.read().strip() != digest(extra)


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    if force or needs_build(extra):
        cmd = [NVCC] + FLAGS + (extra or []) + ["-o", SO] + SRCS
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        with open(STAMP, "w") as f:
            f.write(digest(extra) + "\n")
    return SO


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
