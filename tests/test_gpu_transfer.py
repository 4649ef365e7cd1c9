"""GPU parity of advection and the FLIP transfers (bit-exact: the kernels
keep the reference's FP64 lerps and its summation order)."""
import numpy as np
import pytest

from conftest import golden
from vflip_b200 import scenes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def parts(p):
    return t(p.view(np.uint8))


def unparts(x):
    import oracle

    return x.cpu().numpy().view(oracle.PARTICLE_DTYPE)


OFFS = {"u": (0.5, 0, 0), "v": (0, 0.5, 0), "w": (0, 0, 0.5), "c": (0, 0, 0)}


def test_advect_golden(gpu_solver):
    g = golden("advect")
    ni, nj, nk = (int(x) for x in g["dims"])
    for name, offs in OFFS.items():
        out = gpu_solver[0].advect_rk2_linear(ni, nj, nk, float(g["h"]), float(g["dt"]), t(g["u"]), t(g["v"]),
                                              t(g["w"]), t(g["in_" + name]), offs)
        assert np.array_equal(out.cpu().numpy(), g["out_" + name]), name


@pytest.mark.parametrize("dims,dt", [((40, 33, 29), 0.03), ((64, 64, 64), 0.01)])
def test_advect_vs_oracle(gpu_solver, orc, dims, dt):
    ni, nj, nk = dims
    rng = np.random.default_rng(11)
    h = np.float32(1.0 / ni)
    u, v, w = scenes.random_velocity(ni, nj, nk, rng, scale=2.0)
    for name, offs in OFFS.items():
        shape = {"u": (nk, nj, ni + 1), "v": (nk, nj + 1, ni), "w": (nk + 1, nj, ni), "c": (nk, nj, ni)}[name]
        f = rng.standard_normal(shape).astype(np.float32)
        want = orc.advect_rk2(ni, nj, nk, h, dt, u, v, w, f, offs)
        got = gpu_solver[0].advect_rk2_linear(ni, nj, nk, h, dt, t(u), t(v), t(w), t(f), offs).cpu().numpy()
        assert np.array_equal(got, want), name
        # FP32 sampling: the backtraced positions carry FP32 rounding (~1e-6
        # of the grid coordinate), which the N(0,1)-per-cell test fields turn
        # into value differences of up to ~1e-4 of their range
        got32 = gpu_solver[1].advect_rk2_linear(ni, nj, nk, h, dt, t(u), t(v), t(w), t(f), offs).cpu().numpy()
        assert np.max(np.abs(got32 - want)) <= 1e-3 * max(1.0, np.abs(want).max()), name
        assert np.sqrt(np.mean((got32 - want) ** 2)) <= 1e-5 * max(1.0, np.abs(want).max()), name


def test_transfer_golden(gpu_solver):
    g = golden("transfer")
    ni, nj, nk = (int(x) for x in g["dims"])
    h = float(g["h"])
    p = t(g["particles"])
    cells = gpu_solver[1].particle_cells(ni, nj, nk, h, p).cpu().numpy()
    assert np.array_equal(cells, g["cells"])
    outs = gpu_solver[1].particle_to_grid(ni, nj, nk, h, p)
    for c in range(3):
        assert np.array_equal(outs[c][0].cpu().numpy(), g[f"p2g_f{c}"])
        assert np.array_equal(outs[c][1].cpu().numpy(), g[f"p2g_c{c}"])
    gpu_solver[1].particle_from_grid(ni, nj, nk, h, p, t(g["du"]), t(g["dv"]), t(g["dw"]))
    assert np.array_equal(p.cpu().numpy(), g["g2p"])


@pytest.mark.parametrize("dims,n", [((33, 29, 21), 200000), ((64, 64, 64), 8 * 64 ** 3)])
def test_p2g_vs_oracle(gpu_solver, orc, dims, n):
    ni, nj, nk = dims
    rng = np.random.default_rng(13)
    h = np.float32(1.0 / ni)
    if n == 8 * ni * nj * nk:
        p = scenes.jittered_particles(ni, nj, nk, h, 8, rng)
        p["vel"] = rng.standard_normal((len(p), 3)).astype(np.float32)
        rng.shuffle(p)
    else:
        p = scenes.random_particles(ni, nj, nk, h, n, rng, margin=1.0)
    outs = gpu_solver[1].particle_to_grid(ni, nj, nk, h, parts(p))
    for c in range(3):
        f, cf = orc.p2g(ni, nj, nk, h, p, c)
        assert np.array_equal(outs[c][0].cpu().numpy(), f)
        assert np.array_equal(outs[c][1].cpu().numpy(), cf)


@pytest.mark.parametrize("order", ["shuffled", "by cell"])
def test_p2g_crowded_cells_and_empty(gpu_solver, orc, order):
    """Buckets far beyond 32 particles (2600 in one cell: heapsort; 700 in
    another: a warp's radix sort when shuffled, its runs of consecutive
    indices when the particles come by cell), particles outside the grid,
    and an empty particle set."""
    ni, nj, nk = 6, 5, 4
    h = np.float32(0.2)
    rng = np.random.default_rng(17)
    p = scenes.random_particles(ni, nj, nk, h, 4300, rng, margin=0.0)
    p["pos"][:2600] = (np.array([2.0, 2.0, 1.0]) * h + rng.uniform(-0.4, 0.4, (2600, 3)) * h).astype(np.float32)
    p["pos"][3000:3700] = (np.array([4.0, 1.0, 2.0]) * h + rng.uniform(-0.4, 0.4, (700, 3)) * h).astype(np.float32)
    p["pos"][2600:2700] = -5.0  # outside
    rng.shuffle(p)
    if order == "by cell":
        c = np.clip(np.floor(p["pos"] / h + 0.5).astype(np.int64), 0, [ni - 1, nj - 1, nk - 1])
        p = p[np.argsort(c[:, 0] + ni * (c[:, 1] + nj * c[:, 2]), kind="stable")]
    outs = gpu_solver[1].particle_to_grid(ni, nj, nk, h, parts(p))
    for c in range(3):
        f, cf = orc.p2g(ni, nj, nk, h, p, c)
        assert np.array_equal(outs[c][0].cpu().numpy(), f)
        assert np.array_equal(outs[c][1].cpu().numpy(), cf)
    empty = torch.zeros((0, 40), dtype=torch.uint8, device=DEV)
    outs = gpu_solver[1].particle_to_grid(ni, nj, nk, h, empty)
    for c in range(3):
        assert torch.all(outs[c][0] == 0) and torch.all(outs[c][1] == np.float32(1e-5))


def test_p2g_dense_tiles_vs_oracle(gpu_solver, orc):
    """A blob of 110 000 particles over a few cells: the tiles around it hold
    many shared-memory chunks and keep their nodes' sums in shared memory
    between chunks."""
    ni, nj, nk = 12, 10, 9
    h = np.float32(1.0 / 16)
    rng = np.random.default_rng(31)
    p = scenes.random_particles(ni, nj, nk, h, 130000, rng, margin=0.5)
    p["pos"][:110000] = (np.array([5.0, 4.0, 4.0]) * h + rng.uniform(-1.5, 1.5, (110000, 3)) * h).astype(np.float32)
    rng.shuffle(p)
    outs = gpu_solver[1].particle_to_grid(ni, nj, nk, h, parts(p))
    for c in range(3):
        f, cf = orc.p2g(ni, nj, nk, h, p, c)
        assert np.array_equal(outs[c][0].cpu().numpy(), f)
        assert np.array_equal(outs[c][1].cpu().numpy(), cf)


@pytest.mark.parametrize("flip", [1.0, 0.95, 0.0])
def test_g2p_vs_oracle(gpu_solver, orc, flip):
    ni, nj, nk = 37, 31, 23
    rng = np.random.default_rng(19)
    h = np.float32(1.0 / ni)
    p = scenes.random_particles(ni, nj, nk, h, 100000, rng, margin=2.0)
    du, dv, dw = scenes.random_velocity(ni, nj, nk, rng)
    un, vn, wn = scenes.random_velocity(ni, nj, nk, rng)
    want = orc.g2p(ni, nj, nk, h, p, du, dv, dw, un, vn, wn, flip_ratio=flip)
    x = parts(p)
    gpu_solver[1].particle_from_grid(ni, nj, nk, h, x, t(du), t(dv), t(dw), t(un), t(vn), t(wn), flip_ratio=flip)
    assert np.array_equal(x.cpu().numpy(), want.view(np.uint8))


def test_delta_and_bricks(gpu_solver, orc):
    rng = np.random.default_rng(23)
    a = rng.standard_normal((9, 10, 13)).astype(np.float32)
    b = rng.standard_normal((9, 10, 13)).astype(np.float32)
    assert np.array_equal(gpu_solver[1].delta(t(a), t(b)).cpu().numpy(), orc.delta(a, b))
    br = gpu_solver[1].linear_to_bricks(13, 10, 9, t(a))
    assert br.numel() == 16 * 16 * 16
    # brick index of Buffer3D (fluid_buffer3D.h:186-202)
    i, j, k = 11, 9, 7
    idx = ((((k >> 3) * 2 * 2) + (j >> 3) * 2 + (i >> 3)) << 9) + ((k & 7) << 6) + ((j & 7) << 3) + (i & 7)
    assert float(br[idx]) == a[k, j, i]
    back = gpu_solver[1].bricks_to_linear(13, 10, 9, br)
    assert np.array_equal(back.cpu().numpy(), a)


def test_advect_pair_matches_single(gpu_solver, orc):
    """Two cell-centred fields advected along one shared backtrace equal two
    separate advections (and the oracle)."""
    ni, nj, nk = 48, 40, 36
    rng = np.random.default_rng(29)
    h = np.float32(1.0 / 64)
    u, v, w = scenes.random_velocity(ni, nj, nk, rng, scale=2.0)
    f = rng.standard_normal((nk, nj, ni)).astype(np.float32)
    g = rng.standard_normal((nk, nj, ni)).astype(np.float32)
    a, b = gpu_solver[0].advect_rk2_linear2(ni, nj, nk, h, 0.02, t(u), t(v), t(w), t(f), t(g), (0, 0, 0))
    assert np.array_equal(a.cpu().numpy(), orc.advect_rk2(ni, nj, nk, h, 0.02, u, v, w, f, (0, 0, 0)))
    assert np.array_equal(b.cpu().numpy(), orc.advect_rk2(ni, nj, nk, h, 0.02, u, v, w, g, (0, 0, 0)))


def _flip_scene(ni, nj, nk, seed, n_particles):
    rng = np.random.default_rng(seed)
    h = np.float32(1.0 / max(ni, nj, nk))
    phi = scenes.random_phi(ni, nj, nk, h, rng, n_spheres=2)
    u, v, w = scenes.random_velocity(ni, nj, nk, rng, scale=0.5)
    p = scenes.random_particles(ni, nj, nk, h, n_particles, rng)
    return h, phi, u, v, w, p


@pytest.mark.parametrize("dims,dt,n", [((12, 10, 9), 0.02, 5000), ((32, 24, 20), 0.05, 60000)])
def test_advect_flip_bit_exact(gpu_solver, orc, dims, dt, n):
    ni, nj, nk = dims
    h, phi, u, v, w, p = _flip_scene(ni, nj, nk, 5, n)
    x = t(p.view(np.uint8))
    gpu_solver[1].advect_flip(ni, nj, nk, h, x, t(u), t(v), t(w), t(phi), dt)
    want = orc.advect_flip(ni, nj, nk, h, p, u, v, w, phi, dt)
    assert np.array_equal(x.cpu().numpy(), want.view(np.uint8))


@pytest.mark.parametrize("dims,n,seed", [((9, 8, 7), 1500, 3), ((24, 20, 16), 40000, 11), ((16, 16, 16), 0, 2)])
def test_reorder_flip_bit_exact(gpu_solver, orc, dims, n, seed):
    """Same counter-based draws as the oracle: the whole reseeded set is equal
    byte for byte (kept particles in cell order, new ones, solid filter)."""
    ni, nj, nk = dims
    h, phi, u, v, w, p = _flip_scene(ni, nj, nk, 9, max(n, 1))
    p = p[:n]
    got = gpu_solver[1].reorder_flip(ni, nj, nk, h, t(p.view(np.uint8)) if n else torch.empty(0, dtype=torch.uint8,
                                                                                                   device=DEV),
                                     t(u), t(v), t(w), t(phi), seed=seed).cpu().numpy()
    want = orc.reorder_flip(ni, nj, nk, h, p, u, v, w, phi, seed=seed)
    assert got.size == want.size * 40 and np.array_equal(got, want.view(np.uint8))


def test_reorder_flip_crowded_cells(gpu_solver, orc):
    """Reseeding keeps the first particles of each bucket in index order:
    buckets of 2500 (heapsort) and 900 (a warp's radix sort) particles."""
    ni, nj, nk = 9, 8, 7
    h, phi, u, v, w, p = _flip_scene(ni, nj, nk, 21, 5000)
    rng = np.random.default_rng(4)
    p["pos"][:2500] = (np.array([4.0, 4.0, 3.0]) * h + rng.uniform(-0.45, 0.45, (2500, 3)) * h).astype(np.float32)
    p["pos"][2500:3400] = (np.array([2.0, 5.0, 4.0]) * h + rng.uniform(-0.45, 0.45, (900, 3)) * h).astype(np.float32)
    rng.shuffle(p)
    got = gpu_solver[1].reorder_flip(ni, nj, nk, h, t(p.view(np.uint8)), t(u), t(v), t(w), t(phi), seed=5)
    want = orc.reorder_flip(ni, nj, nk, h, p, u, v, w, phi, seed=5)
    assert np.array_equal(got.cpu().numpy(), want.view(np.uint8))


def test_reorder_flip_capacity(gpu_solver):
    from vflip_b200._lib import VflipError

    ni = nj = nk = 8
    h, phi, u, v, w, p = _flip_scene(ni, nj, nk, 4, 100)
    with pytest.raises(VflipError):
        gpu_solver[1].reorder_flip(ni, nj, nk, h, t(p.view(np.uint8)), t(u), t(v), t(w), t(phi), capacity=10)


# ---- nested subdomain particle transfers (bit-exact)

def test_subdomain_golden(gpu_solver):
    import oracle

    g = golden("subdomain")
    s = gpu_solver[1]
    ni, nj, nk = (int(x) for x in g["dims"])
    h, bmin = float(g["h"]), g["bmin"]
    p = t(g["particles"])
    assert np.array_equal(s.sub_particle_cells(ni, nj, nk, h, bmin, p).cpu().numpy(), g["cells"])
    outs = s.sub_particle_to_grid(ni, nj, nk, h, bmin, p)
    for c in range(3):
        assert np.array_equal(outs[c][0].cpu().numpy().view(np.uint32), g[f"p2g_f{c}"].view(np.uint32)), c
        assert np.array_equal(outs[c][1].cpu().numpy().view(np.uint32), g[f"p2g_c{c}"].view(np.uint32)), c
    s.sub_particle_from_grid(ni, nj, nk, h, bmin, p, t(g["du"]), t(g["dv"]), t(g["dw"]))
    assert np.array_equal(p.cpu().numpy(), g["g2p"])
    r = s.sub_reorder_flip(ni, nj, nk, h, bmin, t(g["jittered"]), t(g["du"]), t(g["dv"]), t(g["dw"]), t(g["phi"]))
    assert np.array_equal(r.cpu().numpy(), g["reorder"])
    assert oracle.PARTICLE_DTYPE.itemsize == 40


@pytest.mark.parametrize("dims,n", [((24, 20, 22), 60000), ((40, 36, 32), 8 * 40 * 36 * 32)])
def test_subdomain_vs_oracle(gpu_solver, orc, dims, n):
    """Hash, widened P2G, G2P and seeded reseeding of a subdomain whose
    origin is off zero, with particles outside it: the GPU equals the oracle
    byte for byte (the reseeding draws from the same counter-based hash)."""
    ni, nj, nk = dims
    rng = np.random.default_rng(73)
    h = np.float32(1.0 / 64)
    bmin = np.array([0.31, 0.22, 0.27], np.float32)
    if n == 8 * ni * nj * nk:
        p = scenes.jittered_particles(ni, nj, nk, h, 8, rng)
    else:
        p = scenes.random_particles(ni, nj, nk, h, n, rng, margin=3.0)
    p["pos"] += bmin
    s = gpu_solver[1]
    tp = t(p.view(np.uint8))
    assert np.array_equal(s.sub_particle_cells(ni, nj, nk, h, bmin, tp).cpu().numpy(),
                          orc.sub_hash(ni, nj, nk, h, bmin, p))
    outs = s.sub_particle_to_grid(ni, nj, nk, h, bmin, tp)
    for c in range(3):
        f, cf = orc.sub_p2g(ni, nj, nk, h, bmin, p, c)
        assert np.array_equal(outs[c][0].cpu().numpy().view(np.uint32), f.view(np.uint32)), c
        assert np.array_equal(outs[c][1].cpu().numpy().view(np.uint32), cf.view(np.uint32)), c
    du, dv, dw = scenes.random_velocity(ni, nj, nk, rng)
    s.sub_particle_from_grid(ni, nj, nk, h, bmin, tp, t(du), t(dv), t(dw))
    want = orc.sub_g2p(ni, nj, nk, h, bmin, p, du, dv, dw)
    assert np.array_equal(tp.cpu().numpy(), want.view(np.uint8))
    phi = scenes.random_phi(ni, nj, nk, h, rng, n_spheres=3)
    sparse = p[: len(p) // 3]
    r = s.sub_reorder_flip(ni, nj, nk, h, bmin, t(sparse.view(np.uint8)), t(du), t(dv), t(dw), t(phi), seed=5)
    want = orc.sub_reorder_flip(ni, nj, nk, h, bmin, sparse, du, dv, dw, phi, seed=5)
    assert np.array_equal(r.cpu().numpy(), want.view(np.uint8))
