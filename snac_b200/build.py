"""Build libsnac_b200.so in-tree with nvcc for sm_100a.

    python -m snac_b200.build          # rebuild if a source changed
    python -m snac_b200.build --force

The library is one CUDA translation unit compiled with -fmad=false so that
every kernel rounds like the reference's x86-64 build (see csrc/snac_device.cuh).
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsnac_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(CSRC, "*.h")) +
                  [os.path.join(ROOT, "include", "snac_gpu.h")])


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in sources())


def build(force: bool = False, verbose: bool = False, defines=(), out: str = LIB) -> str:
    if not force and not stale() and out == LIB:
        return LIB
    cmd = [nvcc(), *ARCH, *["-D" + d for d in defines], "-lineinfo", "-O3", "-fmad=false", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
           "-shared", "-I" + os.path.join(ROOT, "include"), "-o", out + ".tmp",
           os.path.join(CSRC, "snac_api.cu")]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)
    return out


def ensure_built() -> str:
    return build(force=False)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
