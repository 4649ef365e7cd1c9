"""Entry points and kernel variants that must agree with the ones they stand for:
  * the one-call u, v, w advection gives the three single calls' bits;
  * the plane-marching PCG SpMV gives the column kernel's iterations and,
    up to the grouping of its s.q partial sums, its solution;
  * the one-CTA V-cycle tail gives the per-level launches' bits;
  * the tiled sweep of the small levels gives the marching sweeps' bits;
  * the two-CTA register-carry sweep of rows <= 128 cells gives the plain
    fused kernel's bits;
  * the projection's PCG, which reads the FP32 copies of the couplings it
    assembled, gives the bits of the same solve on the FP64 operator."""
import numpy as np
import pytest

from vflip_b200 import scenes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def smooth_velocity(ni, nj, nk, amp, seed):
    rng = np.random.default_rng(seed)
    out = []
    for sh in scenes.face_shapes(ni, nj, nk):
        k, j, i = np.meshgrid(*(np.arange(x, dtype=np.float32) for x in sh), indexing="ij")
        ph = rng.uniform(0, 6.3, 3)
        out.append((amp * np.sin(0.21 * i + ph[0]) * np.cos(0.17 * j + ph[1]) * np.sin(0.13 * k + ph[2])).astype(
            np.float32))
    return out


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("dims", [(40, 36, 33), (1, 9, 70)])
def test_velocity_advection_one_call(prec, dims):
    from vflip_b200.solver import Solver

    ni, nj, nk = dims
    h = np.float32(1.0 / max(dims))
    U, V, W = (t(x) for x in smooth_velocity(ni, nj, nk, 2.0, seed=5))
    with Solver(precision=prec) as s:
        got = s.advect_velocity_rk2_linear(ni, nj, nk, h, 0.03, U, V, W)
        for name, f, o, g in zip("uvw", (U, V, W), ((0.5, 0, 0), (0, 0.5, 0), (0, 0, 0.5)), got):
            assert torch.equal(g, s.advect_rk2_linear(ni, nj, nk, h, 0.03, U, V, W, f, o)), name


@pytest.mark.parametrize("prec", [1, 2, 0])
def test_plane_spmv_matches_column_kernel(prec):
    from vflip_b200.solver import Solver

    ni, nj, nk = 128, 30, 22
    pr = scenes.projection_problem(ni, nj, nk, seed=9, inflow=True)
    st, rhs = None, None
    res = []
    for k in (0, 1):
        with Solver(precision=prec, spmv_kernel=k) as s:
            if st is None:
                st, rhs = s.assemble(pr["ni"], pr["nj"], pr["nk"], pr["h"], pr["U_in"], t(pr["phi"]), t(pr["bdesc"]),
                                     t(pr["us"]), t(pr["vs"]), t(pr["ws"]), t(pr["u"]), t(pr["v"]), t(pr["w"]))
            ok, x, stats = s.amgpcg_solve(st, rhs, 1e-6, 100)
            assert ok
            res.append((x.clone(), stats.iterations))
    (a, ia), (b, ib) = res
    assert ia == ib
    assert float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)) < (1e-10 if prec == 0 else 1e-5)


@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("dims,direct", [((64, 64, 64), 0), ((80, 72, 64), 0), ((64, 64, 64), 1),
                                         ((128, 96, 72), 0)])
def test_vcycle_tail_matches_per_level_launches(prec, dims, direct):
    """The levels from the first one of <= 4096 cells down run in one CTA
    (coarse_tail 0); one launch per sweep (coarse_tail 1) gives the same
    V-cycle bit for bit, with the FP64 direct coarsest solve or with the
    coarsest sweeps (coarsest_solver 1), and so the same solve."""
    from vflip_b200.solver import Solver

    ni, nj, nk = dims
    pr = scenes.projection_problem(ni, nj, nk, seed=11, inflow=True, solid_velocity=True)
    st = rhs = None
    out = []
    for tail in (0, 1):
        with Solver(precision=prec, coarse_tail=tail, coarsest_solver=direct) as s:
            if st is None:
                st, rhs = s.assemble(ni, nj, nk, pr["h"], pr["U_in"], t(pr["phi"]), t(pr["bdesc"]), t(pr["us"]),
                                     t(pr["vs"]), t(pr["ws"]), t(pr["u"]), t(pr["v"]), t(pr["w"]))
            z = s.vcycle(st, rhs).clone()
            ok, x, stats = s.amgpcg_solve(st, rhs, 1e-6, 100)
            assert ok
            out.append((z, x.clone(), stats.iterations))
    (za, xa, ia), (zb, xb, ib) = out
    assert torch.equal(za, zb)
    assert torch.equal(xa, xb) and ia == ib


@pytest.mark.parametrize("prec,loop", [(1, 0), (2, 0), (1, 1)])
def test_projection_spmv_on_fp32_couplings(prec, loop):
    """vflip_project's outer PCG reads the FP32 fine operator's couplings
    (exact: the assembly writes every coupling as a float value) where
    vflip_amgpcg_solve on the same FP64 operator reads the FP64 ones: the
    same pressure bit for bit, and the same iterations."""
    from vflip_b200.solver import Solver

    ni, nj, nk = 128, 64, 48
    pr = scenes.projection_problem(ni, nj, nk, seed=13, inflow=True, solid_velocity=True)
    with Solver(precision=prec, pcg_loop=loop) as s:
        args = [t(pr[k]) for k in ("phi", "bdesc", "us", "vs", "ws", "u", "v", "w")]
        st, rhs = s.assemble(ni, nj, nk, pr["h"], pr["U_in"], *[a.clone() for a in args])
        ok1, x1, st1 = s.amgpcg_solve(st, rhs, 1e-6, 100)
        ok2, p2, st2 = s.project(ni, nj, nk, pr["h"], pr["U_in"], *args)
        assert ok1 and ok2 and st1.iterations == st2.iterations
        assert torch.equal(x1, p2)


@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("dims", [(128, 128, 128), (72, 40, 36), (64, 48, 17)])
def test_tiled_sweep_matches_marching_sweeps(prec, dims):
    """Levels of <= 64^3 cells sweep as independent halo tiles; with the tiles
    off (tile_sweep_max_cells -1) every level marches: the same V-cycle bit
    for bit (ragged last tiles on every axis included) and the same solve."""
    from vflip_b200.solver import Solver

    ni, nj, nk = dims
    pr = scenes.projection_problem(ni, nj, nk, seed=17, inflow=True, solid_velocity=True)
    st = rhs = None
    out = []
    for cells in (0, -1):
        with Solver(precision=prec, tile_sweep_max_cells=cells) as s:
            if st is None:
                st, rhs = s.assemble(ni, nj, nk, pr["h"], pr["U_in"], t(pr["phi"]), t(pr["bdesc"]), t(pr["us"]),
                                     t(pr["vs"]), t(pr["ws"]), t(pr["u"]), t(pr["v"]), t(pr["w"]))
            z = s.vcycle(st, rhs).clone()
            ok, x, stats = s.amgpcg_solve(st, rhs, 1e-6, 100)
            assert ok
            out.append((z, x.clone(), stats.iterations))
    (za, xa, ia), (zb, xb, ib) = out
    assert torch.equal(za, zb)
    assert torch.equal(xa, xb) and ia == ib


@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("dims", [(128, 96, 72), (100, 64, 50)])
def test_narrow_carry_sweep_matches_plain_kernel(prec, dims):
    """Levels whose rows hold 68..128 cells sweep with the 256-thread,
    two-CTA-per-SM register-carry kernel (the fine level here, with its
    fused prolongation and z.r variants); the plain fused kernel
    (sweep_kernel 1) gives the same V-cycle and the same solve."""
    from vflip_b200.solver import Solver

    ni, nj, nk = dims
    pr = scenes.projection_problem(ni, nj, nk, seed=19, inflow=True, solid_velocity=True)
    st = rhs = None
    out = []
    for kern in (0, 1):
        with Solver(precision=prec, sweep_kernel=kern, tile_sweep_max_cells=-1) as s:
            if st is None:
                st, rhs = s.assemble(ni, nj, nk, pr["h"], pr["U_in"], t(pr["phi"]), t(pr["bdesc"]), t(pr["us"]),
                                     t(pr["vs"]), t(pr["ws"]), t(pr["u"]), t(pr["v"]), t(pr["w"]))
            z = s.vcycle(st, rhs).clone()
            ok, x, stats = s.amgpcg_solve(st, rhs, 1e-6, 100)
            assert ok
            out.append((z, x.clone(), stats.iterations))
    (za, xa, ia), (zb, xb, ib) = out
    assert torch.equal(za, zb)
    assert ia == ib
