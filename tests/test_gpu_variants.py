"""Entry points and kernel variants that must agree with the ones they stand for:
  * the one-call u, v, w advection gives the three single calls' bits;
  * the node-specialised RK2 advection gives the general kernel's bits;
  * the plane-marching PCG SpMV gives the column kernel's iterations and,
    up to the grouping of its s.q partial sums, its solution;
  * the one-CTA V-cycle tail gives the per-level launches' bits;
  * the tiled sweep of the small levels gives the marching sweeps' bits;
  * the two-CTA register-carry sweep of rows <= 128 cells gives the plain
    fused kernel's bits;
  * the projection's PCG, which reads the FP32 copies of the couplings it
    assembled, gives the bits of the same solve on the FP64 operator;
  * the tiled P2G, on the main grid and on a subdomain's, gives the
    per-node global gather's bits."""
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


@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("dims", [(64, 48, 40), (5, 9, 70), (128, 1, 3)])
def test_node_advection_matches_general_kernel(prec, dims):
    """With h a power of two, the node-specialised RK2 advection
    (advect_kernel 0: the first stage read from the node's neighbours, u, v,
    w in one launch) gives the general per-sample kernel's bits
    (advect_kernel 1) on every lattice and for the field pair, including
    velocities of +0 and -0 and backtraces that leave the grid."""
    from vflip_b200.solver import Solver

    ni, nj, nk = dims
    h = np.float32(1.0 / 64)
    vel = smooth_velocity(ni, nj, nk, 2.0, seed=7)
    for a, z in zip(vel, (0.0, -0.0, 0.0)):
        a[:, :, :2] = z
        a[: max(1, a.shape[0] // 3)] *= -1
    U, V, W = (t(x) for x in vel)
    rng = np.random.default_rng(3)
    rho, temp = (t(rng.standard_normal((nk, nj, ni)).astype(np.float32)) for _ in range(2))
    offs = ((0.5, 0, 0), (0, 0.5, 0), (0, 0, 0.5), (0, 0, 0))
    res = []
    for kern in (0, 1):
        with Solver(precision=prec, advect_kernel=kern) as s:
            got = list(s.advect_velocity_rk2_linear(ni, nj, nk, h, 0.03, U, V, W))
            for f, o in zip((U, V, W), offs):
                got.append(s.advect_rk2_linear(ni, nj, nk, h, 0.03, U, V, W, f, o))
            got += list(s.advect_rk2_linear2(ni, nj, nk, h, 0.03, U, V, W, rho, temp, offs[3]))
            res.append(got)
    for i, (a, b) in enumerate(zip(*res)):
        assert torch.equal(a.view(torch.int32), b.view(torch.int32)), i


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


def _p2g_cases():
    rng = np.random.default_rng(23)
    out = []
    # 8 particles per cell, shuffled: every tile stages its buckets
    ni, nj, nk = 41, 35, 30
    h = np.float32(1.0 / ni)
    p = scenes.jittered_particles(ni, nj, nk, h, 8, rng)
    p["vel"] = rng.standard_normal((len(p), 3)).astype(np.float32)
    rng.shuffle(p)
    out.append(("jittered", (ni, nj, nk), h, p, (0, 1, 2)))
    # a blob of 40000 particles in a few cells: its tiles hold more than fit
    # in shared memory and stage them in chunks; some particles outside
    ni, nj, nk = 24, 20, 16
    h = np.float32(0.05)
    p = scenes.random_particles(ni, nj, nk, h, 60000, rng, margin=0.0)
    p["pos"][:40000] = (np.array([9.0, 7.0, 5.0]) * h + rng.uniform(-1.2, 1.2, (40000, 3)) * h).astype(np.float32)
    p["pos"][40000:40100] = -3.0
    rng.shuffle(p)
    out.append(("dense blob", (ni, nj, nk), h, p, (0, 1, 2)))
    # 120000 in a few cells: beyond 8 chunks, the nodes' sums in shared memory
    q = scenes.random_particles(ni, nj, nk, h, 20000, rng, margin=0.5)
    blob = scenes.random_particles(ni, nj, nk, h, 120000, rng, margin=0.0)
    blob["pos"] = (np.array([15.0, 8.0, 9.0]) * h + rng.uniform(-1.4, 1.4, (120000, 3)) * h).astype(np.float32)
    q = np.concatenate([q, blob])
    rng.shuffle(q)
    out.append(("very dense blob", (ni, nj, nk), h, q, (0, 1, 2)))
    # non-finite velocities (NaN sums wherever the window holds one)
    ni, nj, nk = 30, 26, 22
    h = np.float32(1.0 / 32)
    p = scenes.jittered_particles(ni, nj, nk, h, 4, rng)
    p["vel"] = rng.standard_normal((len(p), 3)).astype(np.float32)
    bad = rng.choice(len(p), 40, replace=False)
    p["vel"][bad[:20], 0] = np.nan
    p["vel"][bad[20:], 2] = np.inf
    out.append(("non-finite", (ni, nj, nk), h, p, (0, 1, 2)))
    # thin grids, one component, and the three spacings the tents take:
    # not a power of two (above), a power of two <= 1, and one above 1
    for dims, comps, hh in (((1, 9, 70), (0, 1, 2), 1.0 / 16), ((70, 1, 3), (1,), 1.0 / 16),
                            ((17, 16, 8), (2,), 1.0 / 16), ((12, 10, 9), (0, 1, 2), 2.0)):
        h = np.float32(hh)
        p = scenes.jittered_particles(*dims, h, 6, rng)
        p["vel"] = rng.standard_normal((len(p), 3)).astype(np.float32)
        rng.shuffle(p)
        out.append((f"{dims} {comps}", dims, h, p, comps))
    return out


def test_tiled_p2g_matches_global_gather():
    """The tiled P2G (8 x 8 x 8 and 8 x 8 x 4 node tiles, particles staged
    in shared memory, every window particle added) gives the per-node global
    gather's bits (p2g_kernel 1): with one chunk per tile, with tiles staged in
    several chunks, with non-finite velocities, on thin grids and for
    single components."""
    from vflip_b200.solver import Solver

    for name, (ni, nj, nk), h, p, comps in _p2g_cases():
        res = []
        for kern in (1, 0, 2, 3):
            with Solver(precision=1, p2g_kernel=kern) as s:
                outs = s.particle_to_grid(ni, nj, nk, h, t(p.view(np.uint8)), components=comps)
                res.append({c: (outs[c][0].view(torch.int32).clone(), outs[c][1].view(torch.int32).clone())
                            for c in comps})
        for r in res[1:]:
            for c in comps:
                assert torch.equal(res[0][c][0], r[c][0]), (name, c)
                assert torch.equal(res[0][c][1], r[c][1]), (name, c)


def test_tiled_subdomain_p2g_matches_global_gather():
    """A subdomain's tiled P2G (tiles near its boundary stage a 4-cell ring;
    nodes within 4 cells of the boundary gather 9^3 buckets with the 4h
    tent, the rest 3^3) gives the global shell and inner-box launches' bits
    (p2g_kernel 1), for the three spacing forms, a dense blob (tiles of
    many chunks, node sums in shared memory) and particles outside the
    subdomain (clamped into its edge buckets)."""
    from vflip_b200.solver import Solver

    rng = np.random.default_rng(29)
    cases = []
    for dims, hh, ppc in (((40, 36, 30), 1.0 / 64, 8), ((27, 22, 19), 0.03, 6), ((18, 13, 21), 2.0, 5)):
        h = np.float32(hh)
        bmin = tuple(np.float32(x) for x in rng.uniform(-1.0, 1.0, 3) * h * 7)
        p = scenes.jittered_particles(*dims, h, ppc, rng)
        p["pos"] += np.array(bmin, np.float32)
        p["vel"] = rng.standard_normal((len(p), 3)).astype(np.float32)
        out = scenes.random_particles(*dims, h, 500, rng, margin=3.0)
        out["pos"] += np.array(bmin, np.float32)
        p = np.concatenate([p, out])
        rng.shuffle(p)
        cases.append((dims, h, bmin, p))
    dims, h, bmin, p = cases[0]
    blob = np.concatenate([p] * 6)[:100000].copy()
    blob["pos"] = (np.array([3.0, 30.0, 12.0]) * h + rng.uniform(-1.5, 1.5, (100000, 3)) * h + bmin).astype(np.float32)
    cases.append((dims, h, bmin, np.concatenate([p, blob])))
    for dims, h, bmin, p in cases:
        res = []
        for kern in (1, 0, 3):
            with Solver(precision=1, p2g_kernel=kern) as s:
                outs = s.sub_particle_to_grid(*dims, h, bmin, t(p.view(np.uint8)))
                res.append([(outs[c][0].view(torch.int32).clone(), outs[c][1].view(torch.int32).clone())
                            for c in range(3)])
        for r in res[1:]:
            for c in range(3):
                assert torch.equal(res[0][c][0], r[c][0]), (dims, h, c)
                assert torch.equal(res[0][c][1], r[c][1]), (dims, h, c)
