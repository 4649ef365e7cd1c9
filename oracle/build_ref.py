#!/usr/bin/env python3
"""Build the reference solver's own CPU code into oracle/_ref/libvflip_ref.so.

Test infrastructure only: the library this makes is the comparison that pins the
oracle restatement (oracle/vflip_oracle.cpp) and the timed "reference" CPU arm
of bench.py.  It is never linked into the product.

Recipe (nothing of the reference is committed; everything written lands in
oracle/_ref/, which git ignores):
  1. copy Smoke_Solver/*.h and the four translation units the hot path needs
     (GeometricLevelGen.cpp, levelset_util.cpp, Smoke_solver3D.cpp,
     sub_domain.cpp) from the reference tree into oracle/_ref/src;
  2. apply two mechanical patches that only make MSVC-2010 code legal C++14
     for g++ (no arithmetic is touched):
       a. Multigrid3D.h:153 - MultiGridSolver3D uses members of its dependent
          base MultiGrid<T> unqualified (two-phase lookup); add using-decls;
       b. Smoke_solver3D.cpp:1516,1517,1533 - rvalue Vec3f bound to a
          non-const reference (MSVC extension); route through an lvalue helper;
  3. compile with the OpenMP stand-in for tbb::parallel_for (oracle/tbb_shim)
     and -ffp-contract=off so no FMA contraction changes rounding, together
     with the extern "C" harness oracle/ref_harness.cpp.

Where vflip_b200/libvflip_gpu.so is built, a second library,
oracle/_ref/libvflip_ref_dropin.so, compiles the same reference sources and
harness with oracle/dropin/AlgebraicMultigrid.h in place of the reference's
AlgebraicMultigrid.h: its ivock::AMGPCGSolve is include/vflip/amgpcg_dropin.hpp,
so SmokeSolver3D::pcg_projection and SubDomainSolver::pcg_projection run
unchanged with their pressure solve on the GPU (the drop-in test).

Usage: python oracle/build_ref.py [--src /path/to/vFLIP] [--force]
The reference tree is --src, else $VFLIP_REF_SRC, else a checkout named
"reference" beside this repository.  Exit status 0 with a message when the
reference tree is absent (nothing built).
"""
import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")


def default_src():
    """The reference tree: $VFLIP_REF_SRC, else ../reference beside the repository."""
    env = os.environ.get("VFLIP_REF_SRC")
    if env:
        return env
    return os.path.normpath(os.path.join(HERE, "..", "..", "reference"))


SRC_OUT = os.path.join(OUT, "src")
LIB = os.path.join(OUT, "libvflip_ref.so")
DROPIN_SRC = os.path.join(OUT, "dropin_src")
DROPIN_LIB = os.path.join(OUT, "libvflip_ref_dropin.so")
REPO = os.path.dirname(HERE)
GPU_LIB_DIR = os.path.join(REPO, "vflip_b200")
TUS = ["GeometricLevelGen.cpp", "levelset_util.cpp", "Smoke_solver3D.cpp", "sub_domain.cpp"]


def _patch(path, old, new, count=1):
    with open(path) as f:
        s = f.read()
    n = s.count(old)
    if n != count:
        raise RuntimeError(f"patch anchor found {n}x (want {count}) in {path}: {old[:60]!r}")
    with open(path, "w") as f:
        f.write(s.replace(old, new))


def build(src_root, force=False):
    ss = os.path.join(src_root, "Smoke_Solver")
    if not os.path.isdir(ss):
        print(f"build_ref: reference tree {ss} absent; oracle/_ref not built")
        return None
    deps = [os.path.join(HERE, "ref_harness.cpp"), os.path.abspath(__file__)]
    if (not force and os.path.exists(LIB)
            and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps)):
        return LIB
    os.makedirs(SRC_OUT, exist_ok=True)
    for fn in os.listdir(ss):
        if fn.endswith(".h") or fn in TUS:
            shutil.copyfile(os.path.join(ss, fn), os.path.join(SRC_OUT, fn))
    # (a) dependent-base members
    _patch(os.path.join(SRC_OUT, "Multigrid3D.h"),
           "class MultiGridSolver3D: public MultiGrid<T>\n{\npublic:\n",
           "class MultiGridSolver3D: public MultiGrid<T>\n{\npublic:\n"
           "\tusing MultiGrid<T>::xk; using MultiGrid<T>::bk; using MultiGrid<T>::rk;"
           " using MultiGrid<T>::xk_new; using MultiGrid<T>::systemk; using MultiGrid<T>::m_max_level;\n")
    # (b) rvalue -> non-const lvalue reference (seedHalo / seed_ghost, never called here)
    sp = os.path.join(SRC_OUT, "Smoke_solver3D.cpp")
    _patch(sp, "sub_domain.is_halo(Vec3f(i,j,k)*_hx, 2.0f*_hx)",
           "sub_domain.is_halo(vflip_lvalue(Vec3f(i,j,k)*_hx), 2.0f*_hx)")
    _patch(sp, "sub_domain.is_in2(Vec3f(i,j,k)*_hx)",
           "sub_domain.is_in2(vflip_lvalue(Vec3f(i,j,k)*_hx))")
    _patch(sp, "get_solid_phi(Vec3f(i,j,k)*sub_domain._hx + sub_domain.bmin)",
           "get_solid_phi(vflip_lvalue(Vec3f(i,j,k)*sub_domain._hx + sub_domain.bmin))")
    with open(os.path.join(SRC_OUT, "vflip_lvalue.h"), "w") as f:
        f.write("#pragma once\n#include <climits>\n#include <cstring>\n"
                "template <class T> T& vflip_lvalue(T&& v) { return v; }\n")
    cmd = ["g++", "-O2", "-fopenmp", "-std=c++14", "-fpermissive", "-ffp-contract=off",
           "-fPIC", "-shared", "-w",
           "-include", os.path.join(SRC_OUT, "vflip_lvalue.h"),
           "-I", os.path.join(HERE, "tbb_shim"), "-I", SRC_OUT,
           os.path.join(HERE, "ref_harness.cpp")] + [os.path.join(SRC_OUT, t) for t in TUS] + [
           "-o", LIB]
    subprocess.check_call(cmd)
    return LIB


def build_dropin(force=False):
    """The reference sources (patched copy in oracle/_ref/src) with the GPU
    drop-in as their AMGPCGSolve, linked against libvflip_gpu.so."""
    if not os.path.isdir(SRC_OUT) or not os.path.exists(os.path.join(GPU_LIB_DIR, "libvflip_gpu.so")):
        return None
    shim = os.path.join(HERE, "dropin", "AlgebraicMultigrid.h")
    deps = [os.path.join(HERE, "ref_harness.cpp"), os.path.abspath(__file__), shim, LIB,
            os.path.join(REPO, "include", "vflip", "amgpcg_dropin.hpp"), os.path.join(REPO, "include", "vflip.h")]
    if (not force and os.path.exists(DROPIN_LIB)
            and all(os.path.getmtime(DROPIN_LIB) >= os.path.getmtime(d) for d in deps)):
        return DROPIN_LIB
    # a separate copy: the units include "AlgebraicMultigrid.h" with quotes,
    # which finds the file beside them first
    os.makedirs(DROPIN_SRC, exist_ok=True)
    for fn in os.listdir(SRC_OUT):
        shutil.copyfile(os.path.join(SRC_OUT, fn), os.path.join(DROPIN_SRC, fn))
    shutil.copyfile(shim, os.path.join(DROPIN_SRC, "AlgebraicMultigrid.h"))
    cmd = ["g++", "-O2", "-fopenmp", "-std=c++14", "-fpermissive", "-ffp-contract=off",
           "-fPIC", "-shared", "-w", "-DVFLIP_REF_DROPIN", "-Wl,-Bsymbolic",
           "-include", os.path.join(DROPIN_SRC, "vflip_lvalue.h"),
           "-I", os.path.join(HERE, "tbb_shim"), "-I", DROPIN_SRC, "-I", os.path.join(REPO, "include"),
           os.path.join(HERE, "ref_harness.cpp")] + [os.path.join(DROPIN_SRC, t) for t in TUS] + [
           "-L", GPU_LIB_DIR, "-l:libvflip_gpu.so", "-Wl,-rpath,$ORIGIN/../../vflip_b200", "-o", DROPIN_LIB]
    subprocess.check_call(cmd)
    return DROPIN_LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=None, help="the vFLIP source tree (default: $VFLIP_REF_SRC or ../reference)")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    lib = build(a.src or default_src(), a.force)
    print(lib or "not built")
    if lib:
        print(build_dropin(a.force) or "drop-in build skipped (libvflip_gpu.so not built)")
    sys.exit(0)
