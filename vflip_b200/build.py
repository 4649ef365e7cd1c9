"""Builds libvflip_gpu.so in-tree from vflip_b200/csrc with nvcc for sm_100a.

    python -m vflip_b200.build [--force] [--verbose]

Each csrc/*.cu is one translation unit (vflip_capi.cu: the solver, projection
and transfer kernels; unet_capi.cu: the learned preconditioner's network),
compiled in parallel into _build/ and linked into one shared library.
-fmad=false keeps a*b+c rounded twice, as the reference's x86-64 build rounds
it, so kernels that follow the reference's order of operations reproduce its
results bit for bit.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libvflip_gpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

BUILD = os.path.join(HERE, "_build")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC",
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


def units():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(BUILD, exist_ok=True)
    procs, objs = [], []
    for src in units():
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc] + NVCC_FLAGS + list(extra) + ["-I", INCLUDE, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((subprocess.Popen(cmd), cmd))
        objs.append(obj)
    for p, cmd in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, cmd)
    cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC"] + objs + [
        "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
