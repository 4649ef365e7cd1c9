"""vflip_b200 - the vFLIP per-step hot path on NVIDIA B200 (sm_100a).

The compute lives in ``libvflip_gpu.so`` (hand-written CUDA behind the C ABI
in ``include/vflip.h``); this package is a thin host-side mirror of the
reference's solver call surface over that ABI:

    amgpcg_solve(...)      ivock::AMGPCGSolve        (AlgebraicMultigrid.h:189-301)
    project(...)           SmokeSolver3D::pcg_projection (Smoke_solver3D.cpp:945-1202)
    advect_rk2_linear(...) SubDomainSolver::advect_field  (sub_domain.cpp:191-235)
    particle_to_grid(...)  SmokeSolver3D::particle_to_grid (Smoke_solver3D.cpp:1451-1510)
    particle_from_grid(...) SmokeSolver3D::particle_from_grid (Smoke_solver3D.cpp:1398-1406)

Device arrays are torch CUDA tensors (PyTorch provides device memory and
streams only).  There is no CPU fallback: without the built library or a GPU
every compute call raises.
"""
from ._lib import VflipError, lib_path, load  # noqa: F401
from .particles import PARTICLE_BYTES, PARTICLE_DTYPE  # noqa: F401

PREC_FP64 = 0
PREC_FP32 = 1
PREC_MIXED = 2


def __getattr__(name):
    # The solver module needs torch; import it lazily so that the numpy-only
    # helpers (scenes, particles) stay importable without it.
    if name in ("Solver", "SolveStats"):
        from . import solver

        return getattr(solver, name)
    raise AttributeError(name)
