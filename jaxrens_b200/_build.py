"""Compile the CUDA library in-tree for sm_100a.

``python -m jaxrens_b200._build`` (or ``__graft_entry__.build()``) writes
``jaxrens_b200/_lib/libjaxrens_b200.so``.  The translation unit is compiled
with ``-fmad=false``: every fused multiply-add in the kernels is an explicit
intrinsic, which is what makes the arithmetic reproducible by the CPU check.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc", "jr_ns.cu")
DEPS = [
    os.path.join(HERE, "csrc", f)
    for f in ("jr_ns.cu", "jr_rng.cuh", "jr_walk.cuh", "jr_tune.cu")
] + [os.path.join(ROOT, "include", "jaxrens_b200.h")]
OUT = os.path.join(HERE, "_lib", "libjaxrens_b200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC", "-shared",
]


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in DEPS)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    srcs = [SRC] + [p for p in [os.path.join(HERE, "csrc", "jr_tune.cu")] if os.path.exists(p)]
    cmd = ["nvcc", *NVCC_FLAGS, "-o", OUT + ".tmp", *srcs]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
