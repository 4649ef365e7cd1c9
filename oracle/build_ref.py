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

Usage: python oracle/build_ref.py [--src /path/to/reference] [--force]
Exit status 0 with a message when the reference tree is absent (nothing built).
"""
import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SRC_OUT = os.path.join(OUT, "src")
LIB = os.path.join(OUT, "libvflip_ref.so")
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


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default="/root/reference")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    lib = build(a.src, a.force)
    print(lib or "not built")
    sys.exit(0)
