"""Builds the assembler's CUDA library (lib/libfem_alls.so) for sm_100a.

    python build.py            # incremental: rebuilds when a source is newer
    python build.py --force    # always rebuild
    python build.py --ptxas-v  # also print ptxas register / spill / smem use

The library exports only the C ABI declared in include/fem_alls.h.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "lib", "libfem_alls.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + glob.glob(os.path.join(HERE, "csrc", "*.h"))
                  + glob.glob(os.path.join(ROOT, "include", "*.h")))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in sources() + headers())


def build(force: bool = False, ptxas_verbose: bool = False) -> str:
    if not force and not ptxas_verbose and up_to_date():
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cmd = ["nvcc", "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-shared", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(HERE, "csrc"), "-o", LIB + ".tmp", *sources()]
    if ptxas_verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, ptxas_verbose="--ptxas-v" in sys.argv))
