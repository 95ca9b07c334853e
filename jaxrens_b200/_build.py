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
CSRC = os.path.join(HERE, "csrc")
# translation units linked into the one library (each is self-contained)
SRCS = [os.path.join(CSRC, f) for f in ("jr_ns.cu", "jr_pair_ext.cu", "jr_pair_aux.cu", "jr_sw.cu",
                                        "jr_sur.cu", "jr_swda.cu")]


def _deps() -> list[str]:
    hdrs = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cu", ".cuh"))]
    return hdrs + [os.path.join(ROOT, "include", "jaxrens_b200.h")]


OUT = os.path.join(HERE, "_lib", "libjaxrens_b200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC",
]


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(d) > t for d in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every translation unit to an object in parallel, then link."""
    if not force and not _stale():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    objdir = os.path.join(HERE, "_lib", "_obj")
    os.makedirs(objdir, exist_ok=True)
    procs, objs = [], []
    for src in SRCS:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = ["nvcc", *NVCC_FLAGS, "-c", "-o", obj, src]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), file=sys.stderr)
        procs.append((subprocess.Popen(cmd), cmd))
        objs.append(obj)
    failed = [cmd for p, cmd in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    link = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
            "-Xcompiler", "-fPIC", "-o", OUT + ".tmp", *objs]
    subprocess.run(link, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
