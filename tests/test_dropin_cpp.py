"""The header-only C++ drop-in (include/vflip/amgpcg_dropin.hpp): compiles
against a reference-shaped SparseMatrix (CPU) and, on a GPU, solves the
pcg_projection system like the reference solver (checked against the
oracle)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "dropin_main.cpp")


def build(tmp_path):
    from vflip_b200 import build as vb

    vb.build()
    exe = str(tmp_path / "dropin_main")
    libdir = os.path.join(ROOT, "vflip_b200")
    subprocess.check_call(["g++", "-O2", "-std=c++14", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                           "-L", libdir, "-l:libvflip_gpu.so", f"-Wl,-rpath,{libdir}"])
    return exe


def test_dropin_compiles(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_dropin_solves_like_the_reference(tmp_path, orc):
    pytest.importorskip("torch")
    exe = build(tmp_path)
    n = 24
    out = str(tmp_path / "out.bin")
    subprocess.check_call([exe, str(n), out])
    data = np.fromfile(out, np.float64)
    rhs, p, tail = data[:n ** 3], data[n ** 3:2 * n ** 3], data[2 * n ** 3:]
    from vflip_b200 import scenes

    h = np.float32(1.0 / n)
    o = np.ones((n + 1, n + 1, n + 1), np.float32)
    st = scenes.poisson_stencil(n, n, n, h, o[:n, :n, :n + 1], o[:n, :n + 1, :n], o[:n + 1, :n, :n])
    x, ok, res, it = orc.amgpcg(st, rhs.reshape(n, n, n))
    assert bool(tail[0]) == ok and int(tail[1]) == it
    assert np.linalg.norm(p - x.ravel()) <= 1e-11 * np.linalg.norm(x)


def test_nested_step_sequence_compiles_as_c():
    """The coupled time_step sequence (C ABI only, tests/cpp/nested_step.c)
    compiles as C99 against include/vflip.h with warnings as errors."""
    src = os.path.join(ROOT, "tests", "cpp", "nested_step.c")
    subprocess.check_call(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I",
                           os.path.join(ROOT, "include"), src])
