"""The reference's own SmokeSolver3D::pcg_projection and
SubDomainSolver::pcg_projection, compiled from its sources with the
header-only drop-in (include/vflip/amgpcg_dropin.hpp) in place of
AlgebraicMultigrid.h (oracle/_ref/libvflip_ref_dropin.so, made by
oracle/build_ref.py).  The reference's real SparseMatrix assembly
(sparse_matrix.h:13-105, Smoke_solver3D.cpp:945-1120) feeds the GPU solve;
the pressure, the iteration count and the projected velocities match the
reference's CPU solve of the same inputs."""
import numpy as np
import pytest

import oracle
from vflip_b200 import scenes


@pytest.fixture(scope="module")
def dropin():
    d = oracle.reference_dropin()
    if d is None:
        pytest.skip("oracle/_ref/libvflip_ref_dropin.so not built here (needs the reference tree)")
    return d


def test_dropin_library_loads_and_exports(dropin):
    """Loads without a GPU (libvflip_gpu.so resolves through its rpath) and
    exports the reference entry points whose solves go through the drop-in."""
    for name in ("ref_project", "ref_project_subdomain", "ref_amgpcg", "ref_smoke_step", "ref_levels"):
        assert hasattr(dropin.lib, name)
    # the CPU multigrid internals are not in this build: the GPU solve replaces them
    assert not hasattr(dropin.lib, "ref_rbgs")


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("dims,seed", [((24, 22, 20), 3), ((33, 29, 40), 7)])
def test_reference_projection_through_the_dropin(dropin, ref, dims, seed):
    """SmokeSolver3D::pcg_projection (inflow, moving solids, odd non-cubic
    grid): same success flag and iteration count as the reference's CPU
    solve, pressure within 1e-11 relative L2 (the FP64 V-cycle is the
    reference's bit for bit; the PCG's reductions run in another order), and
    the velocity update of the same float arithmetic."""
    pr = scenes.projection_problem(*dims, seed=seed, inflow=True, solid_velocity=True)
    want = ref.project(**pr)
    got = dropin.project(**pr)
    assert got["ok"] == want["ok"] and got["ok"]
    assert got["iterations"] == want["iterations"]
    assert np.array_equal(got["rhs"], want["rhs"]) and np.array_equal(got["stencil"], want["stencil"])
    assert rel(got["pressure"], want["pressure"]) <= 1e-11
    for k in ("u", "v", "w"):
        scale = float(np.abs(want[k]).max())
        assert np.allclose(got[k], want[k], rtol=0, atol=1e-6 * scale), k


@pytest.mark.gpu
def test_reference_subdomain_projection_through_the_dropin(dropin, ref):
    """SubDomainSolver::pcg_projection (dt-scaled operator, AMGPCGSolve at
    1e-9 / 1000 iterations) with the drop-in: pressure within 1e-9 relative L2
    of the reference's CPU solve, velocities to float rounding."""
    pr = scenes.projection_problem(20, 18, 22, seed=5, solid_velocity=True)
    args = [pr[k] for k in ("ni", "nj", "nk", "h")] + [0.5] + [pr[k] for k in ("phi", "us", "vs", "ws", "u", "v", "w")]
    want = ref.project_subdomain(*args)
    got = dropin.project_subdomain(*args)
    assert np.array_equal(got["rhs"], want["rhs"])
    assert rel(got["pressure"], want["pressure"]) <= 1e-9
    for k in ("u", "v", "w"):
        scale = float(np.abs(want[k]).max())
        assert np.allclose(got[k], want[k], rtol=0, atol=1e-6 * scale), k
