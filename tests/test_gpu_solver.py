"""GPU parity of the MGPCG path (calls go through the C ABI).

Bar: the FP64 path reproduces the oracle (and so the reference) bit for bit
for the hierarchy, the smoother and the V-cycle; the PCG differs only by
the order of the tree reductions of its inner products (rel. L2 <= 1e-11,
same iteration count).  FP32 and mixed precision meet the reduced-precision
tolerance: pressure within 1e-5 relative L2 of the reference solve.
"""
import numpy as np
import pytest

from conftest import REF_HIERARCHY, golden, problem_from_golden
from vflip_b200 import scenes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def four(st7):
    """(7, ...) oracle stencil -> (4, ...) device stencil: diag, +x, +y, +z."""
    return t(np.stack([st7[0], st7[2], st7[4], st7[6]]))


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def cases():
    return [("proj_a", None), ("proj_b", None), ("gen", (37, 33, 29)), ("gen", (64, 48, 40))]


def system(orc, tag, dims, seed=4):
    if tag == "gen":
        pr = scenes.projection_problem(*dims, seed=seed, inflow=True, solid_velocity=True)
    else:
        pr = problem_from_golden(golden(tag))
    out = orc.project(**pr)
    return pr, out


@pytest.mark.parametrize("tag,dims", cases())
def test_levels_bit_exact(gpu_solver, orc, tag, dims):
    _, out = system(orc, tag, dims)
    st = out["stencil"]
    ref_levels = orc.levels(st)
    got = gpu_solver[0].build_levels(four(st))
    assert len(got) == len(ref_levels)
    for g, r in zip(got, ref_levels):
        g = g.cpu().numpy()
        assert np.array_equal(g, np.stack([r[0], r[2], r[4], r[6]]))


@pytest.mark.parametrize("tag,dims", cases())
def test_rbgs_bit_exact(gpu_solver, orc, tag, dims):
    _, out = system(orc, tag, dims)
    st, b = out["stencil"], out["rhs"]
    x0 = np.random.default_rng(3).standard_normal(b.shape)
    want = orc.rbgs(st, b, x0, 3)
    got = gpu_solver[0].rbgs(four(st), t(b), t(x0), 3).cpu().numpy()
    assert np.array_equal(got, want)


@pytest.mark.parametrize("tag,dims", cases())
def test_vcycle_bit_exact_fp64(gpu_solver, orc, tag, dims):
    _, out = system(orc, tag, dims)
    st, b = out["stencil"], out["rhs"]
    want = orc.vcycle(st, b)
    got = gpu_solver[0].vcycle(four(st), t(b)).cpu().numpy()
    assert np.array_equal(got, want)


@pytest.mark.parametrize("prec,tol", [(1, 2e-5), (2, 2e-2)])
def test_vcycle_reduced_precision(gpu_solver, orc, prec, tol):
    _, out = system(orc, "gen", (64, 48, 40))
    st, b = out["stencil"], out["rhs"]
    want = orc.vcycle(st, b)
    got = gpu_solver[prec].vcycle(four(st), t(b)).cpu().numpy()
    assert rel_l2(got, want) < tol


@pytest.mark.parametrize("dims", [(64, 48, 40), (128, 96, 64), (36, 20, 44)])
def test_pipelined_sweep_matches_plain_kernel(gpu_solver, orc, dims):
    """The cp.async-pipelined smoother performs the same FP32 operations in
    the same order as the plain fused kernel: identical V-cycles."""
    _, out = system(orc, "gen", dims)
    st, b = four(out["stencil"]), t(out["rhs"])
    a = gpu_solver[1].vcycle(st, b).cpu().numpy()
    c = gpu_solver["f32_plain"].vcycle(st, b).cpu().numpy()
    assert np.array_equal(a, c)
    # mixed precision: BF16 coarse operators through both smoother kernels
    a = gpu_solver[2].vcycle(st, b).cpu().numpy()
    c = gpu_solver["mix_plain"].vcycle(st, b).cpu().numpy()
    assert np.array_equal(a, c)


@pytest.mark.parametrize("shape", [(1, 0, 0, 1, 0, 0), (2, 0, 0, 1, 0, 0), (3, 0, 0, 1, 0, 0), (2, 2, 2, 2, 0, 0),
                                   (1, 3, 3, 2, 0, 0), (3, 1, 5, 1, 0, 0), (1, 7, 0, 1, 576, 0),
                                   (1, 7, 0, 1, 512, -1), (2, 5, 3, 1, 576, 3), (1, 0, 0, 1, 0, 8)])
def test_tma_smoother_shapes_match_plain_kernel(gpu_solver, orc, shape):
    """Every copy depth / tile shape / CTA size of the TMA smoother gives the
    plain kernel's V-cycle bit for bit (odd plane counts, clipped edge tiles)."""
    from vflip_b200.solver import Solver

    _, out = system(orc, "gen", (64, 40, 37))
    st, b = four(out["stencil"]), t(out["rhs"])
    d, r, z, c, th, pf = shape
    with Solver(precision=1, sweep_kernel=4, smoother_depth=d, smoother_tile_rows=r, smoother_plane_ranges=z,
                smoother_ctas_per_sm=c, smoother_threads=th, smoother_prefetch=pf, **REF_HIERARCHY) as s:
        a = s.vcycle(st, b).cpu().numpy()
    ref = gpu_solver["f32_plain"].vcycle(st, b).cpu().numpy()
    assert np.array_equal(a, ref)


@pytest.mark.parametrize("dims", [(64, 40, 37), (40, 37, 30), (128, 96, 64), (36, 20, 44), (16, 9, 5)])
@pytest.mark.parametrize("depth", [1, 2, 3])
def test_tiled3d_smoother_matches_plain_kernel(gpu_solver, orc, dims, depth):
    """The 3-D-tiled smoother (TMA tensor boxes, partial tiles at every edge,
    plane ranges, fused zero-x / prolongation variants) gives the plain
    kernel's V-cycle bit for bit, FP32 and with BF16 coarse operators."""
    from vflip_b200.solver import Solver

    _, out = system(orc, "gen", dims)
    st, b = four(out["stencil"]), t(out["rhs"])
    for prec, plain in ((1, "f32_plain"), (2, "mix_plain")):
        with Solver(precision=prec, sweep_kernel=2, smoother_depth=depth, **REF_HIERARCHY) as s:
            a = s.vcycle(st, b).cpu().numpy()
        ref = gpu_solver[plain].vcycle(st, b).cpu().numpy()
        assert np.array_equal(a, ref), prec


@pytest.mark.parametrize("dims", [(64, 40, 37), (40, 37, 30), (128, 96, 64), (36, 20, 44), (16, 9, 5), (256, 23, 19),
                                  (32, 70, 9)])
@pytest.mark.parametrize("depth,prefetch", [(1, 0), (2, -1), (3, 4)])
def test_carry_smoother_matches_plain_kernel(gpu_solver, orc, dims, depth, prefetch):
    """The register-carry smoother (one thread per quad for the whole z
    march, neighbours by warp shuffle; fused zero-x / prolongation variants,
    clipped edge tiles, rows spanning one to two warps or several rows per
    warp) gives the plain kernel's V-cycle bit for bit, FP32 and with BF16
    coarse operators."""
    from vflip_b200.solver import Solver

    _, out = system(orc, "gen", dims)
    st, b = four(out["stencil"]), t(out["rhs"])
    for prec, plain in ((1, "f32_plain"), (2, "mix_plain")):
        with Solver(precision=prec, sweep_kernel=3, smoother_depth=depth, smoother_prefetch=prefetch,
                    **REF_HIERARCHY) as s:
            a = s.vcycle(st, b).cpu().numpy()
        ref = gpu_solver[plain].vcycle(st, b).cpu().numpy()
        assert np.array_equal(a, ref), prec


@pytest.mark.parametrize("dims", [(256, 40, 37), (256, 16, 70)])
def test_fixed_layout_carry_smoother_matches_plain_kernel(gpu_solver, orc, dims):
    """The instance compiled for 256-cell rows, 7-row tiles and one copy
    group (the tuned 256^3 fine-level shape) gives the plain kernel's V-cycle
    bit for bit, with its zero-x, prolongation and z.r variants in a solve."""
    from vflip_b200.solver import Solver

    _, out = system(orc, "gen", dims)
    st, b = four(out["stencil"]), t(out["rhs"])
    for prec, plain in ((1, "f32_plain"), (2, "mix_plain")):
        with Solver(precision=prec, sweep_kernel=3, smoother_depth=1, smoother_tile_rows=7, **REF_HIERARCHY) as s:
            a = s.vcycle(st, b).cpu().numpy()
            conv, p, stats = s.amgpcg_solve(st, b, 1e-6, 50)
        ref = gpu_solver[plain].vcycle(st, b).cpu().numpy()
        assert np.array_equal(a, ref), prec
        conv2, p2, stats2 = gpu_solver[plain].amgpcg_solve(st, b, 1e-6, 50)
        assert conv and conv2 and stats.iterations == stats2.iterations


def test_carry_smoother_pcg(gpu_solver, orc):
    """The fused z.r of the last post-sweep (DOT variant) through a full solve."""
    from vflip_b200.solver import Solver

    _, out = system(orc, "gen", (64, 48, 40))
    st, b = four(out["stencil"]), t(out["rhs"])
    with Solver(precision=1, sweep_kernel=3, **REF_HIERARCHY) as s:
        conv, p, stats = s.amgpcg_solve(st, b, 1e-6, 50)
    conv2, p2, stats2 = gpu_solver["f32_plain"].amgpcg_solve(st, b, 1e-6, 50)
    assert conv and conv2 and stats.iterations == stats2.iterations
    assert rel_l2(p.cpu().numpy(), p2.cpu().numpy()) < 1e-6


def test_tiled3d_smoother_pcg(gpu_solver, orc):
    from vflip_b200.solver import Solver

    _, out = system(orc, "gen", (64, 48, 40))
    st, b = four(out["stencil"]), t(out["rhs"])
    with Solver(precision=1, sweep_kernel=2, **REF_HIERARCHY) as s:
        conv, p, stats = s.amgpcg_solve(st, b, 1e-6, 50)
    conv2, p2, stats2 = gpu_solver["f32_plain"].amgpcg_solve(st, b, 1e-6, 50)
    assert conv and conv2 and stats.iterations == stats2.iterations
    assert rel_l2(p.cpu().numpy(), p2.cpu().numpy()) < 1e-6


@pytest.mark.parametrize("prec", [1, 2])
def test_automatic_hierarchy(gpu_solver, orc, prec):
    """FP32/MIXED contexts coarsen to a level of <= 4^3 solved directly in FP64
    by default (an 8^3 level relaxed by 100 sweeps without it): the solve
    reaches the tolerance in no more iterations than with the reference's
    hierarchy and agrees with the reference's pressure."""
    from vflip_b200.solver import Solver

    _, out = system(orc, "gen", (64, 48, 40))
    st, b = out["stencil"], out["rhs"]
    x, ok, res, it = orc.amgpcg(st, b)
    with Solver(precision=prec) as s:
        conv, p, stats = s.amgpcg_solve(four(st), t(b), 1e-6, 50)
    assert conv and stats.residual <= 1e-6 * stats.rhs_norm
    assert stats.levels > 3 and stats.iterations <= it
    assert rel_l2(p.cpu().numpy(), x) < 1e-4


def test_vcycle_golden(gpu_solver):
    g = golden("proj_b")
    got = gpu_solver[0].vcycle(four(g["out_stencil"]), t(g["out_rhs"])).cpu().numpy()
    assert np.array_equal(got, g["vcycle"])


@pytest.mark.parametrize("tag,dims", cases())
def test_pcg_fp64_matches_reference(gpu_solver, orc, tag, dims):
    _, out = system(orc, tag, dims)
    st, b = out["stencil"], out["rhs"]
    x, ok, res, it = orc.amgpcg(st, b)
    conv, p, stats = gpu_solver[0].amgpcg_solve(four(st), t(b), 1e-6, 50)
    assert conv == ok and stats.iterations == it
    assert rel_l2(p.cpu().numpy(), x) < 1e-11
    assert abs(stats.residual - res) <= 1e-9 * abs(stats.rhs_norm)


@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("tag,dims", cases())
def test_pcg_reduced_precision(gpu_solver, orc, prec, tag, dims):
    _, out = system(orc, tag, dims)
    st, b = out["stencil"], out["rhs"]
    x, ok, res, it = orc.amgpcg(st, b)
    conv, p, stats = gpu_solver[prec].amgpcg_solve(four(st), t(b), 1e-6, 50)
    assert conv and ok
    assert stats.residual <= 1e-6 * stats.rhs_norm
    # pressure within 1e-5 relative L2 of the reference solve
    assert rel_l2(p.cpu().numpy(), x) < 1e-5
    assert stats.iterations <= it + 2


def test_csr_drop_in(gpu_solver, orc):
    import oracle

    _, out = system(orc, "proj_b", None)
    st, b = out["stencil"], out["rhs"]
    _, nk, nj, ni = st.shape
    rs, ci, v = oracle.stencil_to_csr(st)
    ok, x, res, it = gpu_solver[0].amgpcg_solve_csr(rs, ci, v, b, 1e-6, 50, ni, nj, nk)
    want, wok, wres, wit = orc.amgpcg(st, b)
    assert ok == wok and it == wit
    assert rel_l2(x, want.ravel()) < 1e-11


def test_csr_rejects_non_7point_and_asymmetric(gpu_solver):
    import oracle
    from vflip_b200 import VflipError

    st = scenes.uniform_laplacian(8, 8, 8)
    rs, ci, v = oracle.stencil_to_csr(st)
    b = np.ones(512)
    bad = ci.copy()
    bad[rs[100] + 1] = 0  # an entry far off the 7-point pattern
    with pytest.raises(VflipError) as e:
        gpu_solver[1].amgpcg_solve_csr(rs, bad, v, b, 1e-6, 50, 8, 8, 8)
    assert e.value.code == -3
    v2 = v.copy()
    row = 9 * 8 + 3 + 64 * 3
    # perturb the +x coupling of one interior row only
    for e_ in range(rs[row], rs[row + 1]):
        if ci[e_] == row + 1:
            v2[e_] *= 1.5
    with pytest.raises(VflipError) as e:
        gpu_solver[1].amgpcg_solve_csr(rs, ci, v2, b, 1e-6, 50, 8, 8, 8)
    assert e.value.code == -4


def test_csr_host_conversion_on_many_threads(gpu_solver):
    """A 96^3 system (rows split over up to 14 host threads in the CSR
    checks and conversion), in the form pcg_projection hands over (zero
    couplings left out): the host-buffer call gives the device-array solve
    bit for bit.  With bad entries in two rows that different threads own,
    the error names the first of them in row order."""
    import re

    import bench
    from vflip_b200 import VflipError

    ni = nj = nk = 96
    pr = scenes.projection_problem(ni, nj, nk, seed=7, inflow=True, solid_velocity=True)
    s = gpu_solver[1]
    keys = ("h", "U_in", "phi", "bdesc", "us", "vs", "ws", "u", "v", "w")
    st, b = s.assemble(ni, nj, nk, *[t(pr[k]) if isinstance(pr[k], np.ndarray) else pr[k] for k in keys])
    rs, ci, v = bench.csr_of_stencil(st.cpu().numpy())
    ok, x, res, it = s.amgpcg_solve_csr(rs, ci, v, b.cpu().numpy(), 1e-6, 50, ni, nj, nk)
    ok2, x2, st2 = s.amgpcg_solve(st, b, 1e-6, 50)
    assert ok and ok2 and it == st2.iterations
    assert np.array_equal(x, x2.cpu().numpy().ravel())
    n = ni * nj * nk
    bad = ci.copy()
    def with_couplings(r):  # the next row with an off-diagonal entry
        while rs[r + 1] - rs[r] < 2:
            r += 1
        return r

    late, early = with_couplings(n - 5 * ni * nj - 7), with_couplings(n // 3 + 11)
    for row in (late, early):
        bad[rs[row] + 1] = (row + 2 * ni * nj + 3) % n  # off the 7-point pattern
    with pytest.raises(VflipError) as e:
        s.amgpcg_solve_csr(rs, bad, v, b.cpu().numpy(), 1e-6, 50, ni, nj, nk)
    assert e.value.code == -3
    assert re.search(rf"row {early} ", str(e.value))


def test_solver_failure_modes(gpu_solver, orc):
    """Zero rhs -> converged in 0 iterations; a NaN in the rhs -> not
    converged with 0 iterations (rho != rho); max_iterations exhausted -> not
    converged, as AlgebraicMultigrid.h:214-300 returns."""
    st = scenes.uniform_laplacian(20, 19, 18)
    s = gpu_solver[0]
    conv, p, stats = s.amgpcg_solve(four(st), t(np.zeros((18, 19, 20))))
    assert conv and stats.iterations == 0 and float(p.abs().max()) == 0.0
    r = np.random.default_rng(2).standard_normal((18, 19, 20))
    r[9, 9, 9] = np.nan
    conv, p, stats = s.amgpcg_solve(four(st), t(r))
    assert not conv and stats.iterations == 0
    r = np.random.default_rng(1).standard_normal((18, 19, 20))
    x, ok, res, it = orc.amgpcg(st, r, 1e-14, 2)
    conv, p, stats = s.amgpcg_solve(four(st), t(r), 1e-14, 2)
    assert not conv and not ok and stats.iterations == it == 2
    assert rel_l2(p.cpu().numpy(), x) < 1e-12


@pytest.mark.parametrize("dims", [(3, 3, 3), (1, 1, 1), (16, 16, 16), (5, 40, 3)])
def test_small_and_single_level_grids(gpu_solver, orc, dims):
    ni, nj, nk = dims
    rng = np.random.default_rng(7)
    st = scenes.uniform_laplacian(ni, nj, nk)
    b = rng.standard_normal((nk, nj, ni))
    b[st[0] == 0] = 0.0
    x, ok, res, it = orc.amgpcg(st, b)
    conv, p, stats = gpu_solver[0].amgpcg_solve(four(st), t(b))
    assert conv == ok and stats.iterations == it
    assert rel_l2(p.cpu().numpy(), x) < 1e-11 or np.abs(x).max() == 0


@pytest.mark.parametrize("prec,tol", [(0, 1e-9), (1, 2e-5), (2, 2e-5)])
def test_projection_matches_reference(gpu_solver, orc, prec, tol):
    for tag in ("proj_a", "proj_b"):
        g = golden(tag)
        pr = problem_from_golden(g)
        u, v, w = t(pr["u"]), t(pr["v"]), t(pr["w"])
        conv, p, stats = gpu_solver[prec].project(pr["ni"], pr["nj"], pr["nk"], pr["h"], pr["U_in"], t(pr["phi"]),
                                                  t(pr["bdesc"]), t(pr["us"]), t(pr["vs"]), t(pr["ws"]), u, v, w)
        assert conv
        assert rel_l2(p.cpu().numpy(), g["out_pressure"]) < tol
        for name, arr in (("u", u), ("v", v), ("w", w)):
            assert rel_l2(arr.cpu().numpy(), g["out_" + name]) < tol, name


def test_assembly_bit_exact(gpu_solver):
    for tag in ("proj_a", "proj_b"):
        g = golden(tag)
        pr = problem_from_golden(g)
        u, v, w = t(pr["u"]), t(pr["v"]), t(pr["w"])
        st, rhs = gpu_solver[1].assemble(pr["ni"], pr["nj"], pr["nk"], pr["h"], pr["U_in"], t(pr["phi"]),
                                         t(pr["bdesc"]), t(pr["us"]), t(pr["vs"]), t(pr["ws"]), u, v, w)
        ref = g["out_stencil"]
        assert np.array_equal(st.cpu().numpy(), np.stack([ref[0], ref[2], ref[4], ref[6]]))
        assert np.array_equal(rhs.cpu().numpy(), g["out_rhs"])
        uw, vw, ww = gpu_solver[1].face_weights(pr["ni"], pr["nj"], pr["nk"], t(pr["phi"]))
        for a, k in ((uw, "uw"), (vw, "vw"), (ww, "ww")):
            assert np.array_equal(a.cpu().numpy(), g["out_" + k])


def test_fraction_inside_zero_corners(gpu_solver, orc):
    """Exact-zero corner patterns on which the reference loops forever: the
    kernel terminates and agrees with the oracle's bounded restatement."""
    ni = nj = nk = 4
    phi = np.ones((nk + 1, nj + 1, ni + 1), np.float32)
    phi[2, 2, :] = 0.0
    phi[1, :, 2] = 0.0
    phi[3, 3, 3] = -1.0
    want = orc.face_weights(ni, nj, nk, 0.25, phi)
    got = gpu_solver[1].face_weights(ni, nj, nk, t(phi))
    for a, b in zip(got, want):
        assert np.array_equal(a.cpu().numpy(), b)


def test_subdomain_projection_matches_reference(gpu_solver):
    """SubDomainSolver::pcg_projection: FP64 at the reference's 1e-9 / 1000
    reproduces the reference's pressure and velocities; the assembly is
    bit-exact."""
    g = golden("proj_sub")
    ni, nj, nk = (int(x) for x in g["dims"])
    h, dt = float(g["h"]), float(g["dt"])
    args = [t(g["in_" + k]) for k in ("phi", "us", "vs", "ws")]
    u, v, w = t(g["in_u"]), t(g["in_v"]), t(g["in_w"])
    conv, p, stats = gpu_solver[0].project_subdomain(ni, nj, nk, h, dt, *args, u, v, w)
    assert conv and stats.residual <= 1e-9 * stats.rhs_norm
    assert rel_l2(p.cpu().numpy(), g["out_pressure"]) < 1e-9
    for name, arr in (("u", u), ("v", v), ("w", w)):
        assert rel_l2(arr.cpu().numpy(), g["out_" + name]) < 1e-9, name
    # FP32 to the projection tolerance of the main domain
    u, v, w = t(g["in_u"]), t(g["in_v"]), t(g["in_w"])
    conv, p, stats = gpu_solver[1].project_subdomain(ni, nj, nk, h, dt, *args, u, v, w, tolerance_factor=1e-6,
                                                     max_iterations=50)
    assert conv
    assert rel_l2(p.cpu().numpy(), g["out_pressure"]) < 1e-4


# ---- FP64 direct solve of the coarsest level (FP32 / mixed V-cycles)

def _dense(st4):
    """Dense FP64 matrix of a (4, nk, nj, ni) stencil (diag, +x, +y, +z)."""
    d, xp, yp, zp = (np.asarray(a, np.float64).ravel() for a in st4)
    _, nk, nj, ni = st4.shape
    n = ni * nj * nk
    A = np.diag(d)
    idx = np.arange(n)
    i, j, k = idx % ni, (idx // ni) % nj, idx // (ni * nj)
    for off, c, ok in ((1, xp, i < ni - 1), (ni, yp, j < nj - 1), (ni * nj, zp, k < nk - 1)):
        r = idx[ok]
        A[r, r + off] = c[ok]
        A[r + off, r] = c[ok]
    return A


@pytest.mark.parametrize("dims", [(8, 8, 8), (7, 9, 6), (12, 5, 8), (16, 6, 5), (4, 4, 4), (6, 5, 4)])
@pytest.mark.parametrize("prec", [1, 2])
def test_coarse_direct_solve_matches_dense_solve(orc, dims, prec):
    """A level small enough to be the whole hierarchy (coarsening stops at
    512 unknowns here): the V-cycle is the coarsest solve, the FP64
    band-Cholesky solve, with its factor read from global memory (8^3,
    12x5x8, 16x6x5) or staged in shared memory (the others).  It agrees with a dense
    FP64 solve of the same system (cells without fluid decoupled, x = 0) to
    the FP32 rounding of its input and output."""
    from vflip_b200.solver import Solver

    _, out = system(orc, "gen", dims)
    st7, b = out["stencil"], out["rhs"]
    st4 = np.stack([st7[0], st7[2], st7[4], st7[6]])
    A = _dense(st4)
    b32 = b.astype(np.float32).astype(np.float64).ravel()
    live = np.diag(A) != 0
    want = np.zeros_like(b32)
    want[live] = np.linalg.solve(A[np.ix_(live, live)], b32[live])
    with Solver(precision=prec, coarsest_solver=2, coarsest_max_unknowns=512) as s:
        x = s.vcycle(four(st7), t(b)).cpu().numpy().astype(np.float64).ravel()
    assert (~live).sum() > 0 and live.sum() > 0 and np.all(x[~live] == 0)
    assert rel_l2(x, want) < 2e-6
    # the automatic choice takes the same path in FP32 / mixed precision
    with Solver(precision=prec, coarsest_max_unknowns=512) as s:
        x0 = s.vcycle(four(st7), t(b)).cpu().numpy().astype(np.float64).ravel()
    assert np.array_equal(x0, x)


def test_coarse_direct_singular_level_falls_back_to_sweeps():
    """A pure-Neumann level (no cell pinned by an open boundary) is
    singular: the factorisation flags it and the red-black sweeps run, so
    the result equals the sweeps-only context bit for bit."""
    from vflip_b200.solver import Solver

    ni, nj, nk = 8, 7, 6
    k, j, i = np.meshgrid(np.arange(nk), np.arange(nj), np.arange(ni), indexing="ij")
    xp = np.where(i < ni - 1, -1.0, 0.0)
    yp = np.where(j < nj - 1, -1.0, 0.0)
    zp = np.where(k < nk - 1, -1.0, 0.0)
    diag = ((i > 0).astype(float) + (i < ni - 1) + (j > 0) + (j < nj - 1) + (k > 0) + (k < nk - 1))
    st = t(np.stack([diag, xp, yp, zp]).astype(np.float64))
    b = np.random.default_rng(3).standard_normal((nk, nj, ni))
    b -= b.mean()
    with Solver(precision=1, coarsest_solver=2, coarsest_max_unknowns=512) as s:
        a = s.vcycle(st, t(b)).cpu().numpy()
    with Solver(precision=1, coarsest_solver=1, coarsest_max_unknowns=512) as s:
        ref = s.vcycle(st, t(b)).cpu().numpy()
    assert np.all(np.isfinite(a)) and np.array_equal(a, ref)


@pytest.mark.parametrize("prec", [1, 2])
def test_coarse_direct_pcg(orc, prec):
    """Full FP32 / mixed solves with the automatic coarsest level (the direct
    solve of a <= 4^3 level) reach the tolerance in no more iterations than
    with 100 sweeps on an 8^3 level and agree with the reference's pressure."""
    from vflip_b200.solver import Solver

    _, out = system(orc, "gen", (64, 48, 40))
    st, b = four(out["stencil"]), t(out["rhs"])
    x_ref, ok, res, it = orc.amgpcg(out["stencil"], out["rhs"])
    with Solver(precision=prec) as s:
        conv, p, stats = s.amgpcg_solve(st, b, 1e-6, 50)
    with Solver(precision=prec, coarsest_solver=1) as s:
        conv2, p2, stats2 = s.amgpcg_solve(st, b, 1e-6, 50)
    assert conv and conv2 and stats.iterations <= stats2.iterations
    assert rel_l2(p.cpu().numpy(), x_ref) < 1e-5
