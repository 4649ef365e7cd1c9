"""Builds libvflip_gpu.so in-tree from vflip_b200/csrc with nvcc for sm_100a.

    python -m vflip_b200.build [--force] [--verbose]

The library is one translation unit (csrc/vflip_capi.cu includes every
kernel header).  -fmad=false keeps a*b+c rounded twice, as the reference's
x86-64 build rounds it, so kernels that follow the reference's order of
operations reproduce its results bit for bit.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libvflip_gpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-shared",
]


def sources():
    out = []
    for fn in sorted(os.listdir(CSRC)):
        if fn.endswith((".cu", ".cuh", ".h")):
            out.append(os.path.join(CSRC, fn))
    out.append(os.path.join(INCLUDE, "vflip.h"))
    return out


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in sources())


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + list(extra) + ["-I", INCLUDE, os.path.join(CSRC, "vflip_capi.cu"), "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
