import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libvflip_gpu.so")


@pytest.fixture(scope="session")
def orc():
    """The oracle restatement (built on demand; gcc is on every box)."""
    import oracle

    # make is a no-op when liboracle.so is newer than its source
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"])
    return oracle.oracle()


@pytest.fixture(scope="session")
def ref():
    import oracle

    r = oracle.reference()
    if r is None:
        pytest.skip("reference library oracle/_ref/libvflip_ref.so not built here")
    return r


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def nested_from_golden():
    """The nested fixture and its subdomain as the dict the oracle and the
    library take (dims, h, bmin, u, v, w, phi)."""
    g = golden("nested")
    sub = dict(dims=tuple(int(x) for x in g["sub_dims"]), h=np.float32(g["sub_h"]), bmin=g["sub_bmin"],
               u=g["sub_u"], v=g["sub_v"], w=g["sub_w"], phi=g["sub_phi"])
    return g, sub


def problem_from_golden(g):
    ni, nj, nk = (int(x) for x in g["dims"])
    pr = dict(ni=ni, nj=nj, nk=nk, h=float(g["h"]), U_in=float(g["U_in"]))
    for k in ("phi", "bdesc", "us", "vs", "ws", "u", "v", "w"):
        pr[k] = g["in_" + k]
    return pr


REF_HIERARCHY = dict(coarse_sweeps=200, coarsest_max_unknowns=4096)


@pytest.fixture(scope="session")
def gpu_solver():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from vflip_b200 import build
    from vflip_b200.solver import Solver

    build.build()
    # the reference's hierarchy (16^3 coarsest level, 200 sweeps) in every
    # precision, so V-cycles compare with the oracle's
    s = {p: Solver(precision=p, **REF_HIERARCHY) for p in (0, 1, 2)}
    s["f32_plain"] = Solver(precision=1, sweep_kernel=1, **REF_HIERARCHY)  # the non-pipelined smoother
    s["mix_plain"] = Solver(precision=2, sweep_kernel=1, **REF_HIERARCHY)
    yield s
    for v in s.values():
        v.close()
