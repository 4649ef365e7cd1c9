"""GPU parity of the grid advection forms of SmokeSolver3D beside the
RK2-linear one (cubic-clamped, RK3) and of the smoke scalars on the doubled
density/temperature grid (gen_heat, add_smokeforce).  FP64 contexts and the
scalar kernels are bit-exact with the oracle and the reference's fixture;
FP32 contexts run the same schemes in FP32 within a stated tolerance."""
import numpy as np
import pytest

from conftest import golden
from vflip_b200 import scenes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
DEV = "cuda:0"

OFFS = {"u": (0.5, 0, 0), "v": (0, 0.5, 0), "w": (0, 0, 0.5), "c": (0, 0, 0)}


def t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def shape_of(name, ni, nj, nk):
    return {"u": (nk, nj, ni + 1), "v": (nk, nj + 1, ni), "w": (nk + 1, nj, ni), "c": (nk, nj, ni)}[name]


def bits(a):
    return np.asarray(a).view(np.uint32)


def test_smoke_golden(gpu_solver):
    from vflip_b200.particles import PARTICLE_DTYPE

    g = golden("smoke")
    s = gpu_solver[0]
    ni, nj, nk = (int(x) for x in g["dims"])
    h, dt = float(g["h"]), float(g["dt"])
    u, v, w = t(g["u"]), t(g["v"]), t(g["w"])
    for name, offs in OFFS.items():
        out = s.advect_cubic_clamp(ni, nj, nk, h, dt, u, v, w, t(g["cubic_in_" + name]), offs)
        assert np.array_equal(bits(out.cpu().numpy()), bits(g["cubic_out_" + name])), name
    fh = h / 2
    r, tp = s.advect_rk3_linear(ni, nj, nk, h, dt, u, v, w, t(g["rho"]), fh, field2=t(g["temp"]))
    assert np.array_equal(bits(r.cpu().numpy()), bits(g["rk3_rho"]))
    assert np.array_equal(bits(tp.cpu().numpy()), bits(g["rk3_temp"]))
    hp = [float(x) for x in g["heat_params"]]
    s.gen_heat(r, tp, fh, hp[0], hp[1], hp[2], hp[3:6], hp[6], hp[7], hp[8])
    assert np.array_equal(bits(r.cpu().numpy()), bits(g["heat_rho"]))
    assert np.array_equal(bits(tp.cpu().numpy()), bits(g["heat_temp"]))
    p = t(g["particles"])
    fp = [float(x) for x in g["force_params"]]
    s.add_smokeforce(p, r, tp, fh, *fp)
    assert np.array_equal(p.cpu().numpy(), g["force_particles"])
    assert len(g["particles"].view(PARTICLE_DTYPE)) == 3000


@pytest.mark.parametrize("dims,dt", [((40, 33, 29), 0.03), ((64, 64, 64), 0.012)])
def test_cubic_clamp_vs_oracle(gpu_solver, orc, dims, dt):
    ni, nj, nk = dims
    rng = np.random.default_rng(17)
    h = np.float32(1.0 / ni)
    u, v, w = scenes.random_velocity(ni, nj, nk, rng, scale=2.0)
    tu, tv, tw = t(u), t(v), t(w)
    for name, offs in OFFS.items():
        f = rng.standard_normal(shape_of(name, ni, nj, nk)).astype(np.float32)
        want = orc.advect_cubic_clamp(ni, nj, nk, h, dt, u, v, w, f, offs)
        got = gpu_solver[0].advect_cubic_clamp(ni, nj, nk, h, dt, tu, tv, tw, t(f), offs).cpu().numpy()
        assert np.array_equal(bits(got), bits(want)), name
        # FP32: positions carry FP32 rounding (values within ~1e-4 of the
        # N(0,1) field), and at the rare node whose cubic value sits within
        # that rounding of the corner range's edge the clamp may pick the
        # other branch (both lie in the corner range), so bound the share of
        # nodes off by more than 1e-3 rather than the maximum
        got32 = gpu_solver[1].advect_cubic_clamp(ni, nj, nk, h, dt, tu, tv, tw, t(f), offs).cpu().numpy()
        scale = max(1.0, np.abs(want).max())
        off = np.abs(got32 - want) > 1e-3 * scale
        assert off.mean() <= 1e-4, (name, off.sum())
        assert np.sqrt(np.mean((got32 - want)[~off] ** 2)) <= 1e-5 * scale, name


def test_velocity_cubic_clamp_one_launch(gpu_solver, orc):
    """SmokeSolver3D::advect: the three components in one launch equal three
    single-field calls of the oracle (bit-exact in FP64)."""
    ni, nj, nk = 24, 20, 18
    rng = np.random.default_rng(19)
    h = np.float32(1.0 / 24)
    u, v, w = scenes.random_velocity(ni, nj, nk, rng, scale=2.5)
    outs = gpu_solver[0].advect_velocity_cubic_clamp(ni, nj, nk, h, 0.04, t(u), t(v), t(w))
    for name, f, got in zip("uvw", (u, v, w), outs):
        want = orc.advect_cubic_clamp(ni, nj, nk, h, 0.04, u, v, w, f, OFFS[name])
        assert np.array_equal(bits(got.cpu().numpy()), bits(want)), name
    with pytest.raises(RuntimeError):
        x = t(u)
        gpu_solver[0].advect_velocity_cubic_clamp(ni, nj, nk, h, 0.04, x, t(v), t(w), outs=(x, outs[1], outs[2]))


@pytest.mark.parametrize("n,dt", [(24, 0.05), (48, 0.02)])
def test_rk3_double_grid_vs_oracle(gpu_solver, orc, n, dt):
    """Density and temperature on the 2n grid at h/2 (and a face grid at h),
    advected along one shared RK3 backtrace."""
    rng = np.random.default_rng(23)
    h = np.float32(1.0 / n)
    u, v, w = scenes.random_velocity(n, n, n, rng, scale=2.0)
    tu, tv, tw = t(u), t(v), t(w)
    fh = float(h) / 2
    rho = rng.random((2 * n,) * 3).astype(np.float32)
    temp = rng.standard_normal((2 * n,) * 3).astype(np.float32)
    want_r = orc.advect_rk3(n, n, n, h, dt, u, v, w, rho, fh)
    want_t = orc.advect_rk3(n, n, n, h, dt, u, v, w, temp, fh)
    r, tp = gpu_solver[0].advect_rk3_linear(n, n, n, h, dt, tu, tv, tw, t(rho), fh, field2=t(temp))
    assert np.array_equal(bits(r.cpu().numpy()), bits(want_r))
    assert np.array_equal(bits(tp.cpu().numpy()), bits(want_t))
    f = rng.standard_normal((n, n, n + 1)).astype(np.float32)
    got = gpu_solver[0].advect_rk3_linear(n, n, n, h, dt, tu, tv, tw, t(f), float(h), (0.5, 0, 0))
    assert np.array_equal(bits(got.cpu().numpy()), bits(orc.advect_rk3(n, n, n, h, dt, u, v, w, f, float(h),
                                                                        (0.5, 0, 0))))
    # FP32: three FP32 stages leave ~1e-7 of position error, which the
    # U(0,1)-per-node field (gradient ~1/fh) turns into ~1e-5 of value
    r32 = gpu_solver[1].advect_rk3_linear(n, n, n, h, dt, tu, tv, tw, t(rho), fh).cpu().numpy()
    assert np.max(np.abs(r32 - want_r)) <= 1e-3
    assert np.sqrt(np.mean((r32 - want_r) ** 2)) <= 3e-5


def test_gen_heat_and_smokeforce_vs_oracle(gpu_solver, orc):
    from vflip_b200.particles import PARTICLE_DTYPE

    n = 40
    rng = np.random.default_rng(29)
    h = np.float32(1.0 / n)
    fh = float(h) / 2
    rho = rng.random((2 * n, 2 * n, 2 * n)).astype(np.float32)
    temp = rng.random(rho.shape).astype(np.float32)
    args = (fh, 0.01, 0.05, 0.2, (0.5, 0.1, 0.5), 0.12, 1.0, 3.0)
    want_r, want_t = orc.gen_heat(rho, temp, *args)
    r, tp = t(rho), t(temp)
    gpu_solver[1].gen_heat(r, tp, *args)
    assert np.array_equal(bits(r.cpu().numpy()), bits(want_r))
    assert np.array_equal(bits(tp.cpu().numpy()), bits(want_t))
    assert (want_r == 1.0).sum() > 100
    p = scenes.random_particles(n, n, n, h, 200000, rng, margin=1.5)
    want = orc.add_smokeforce(p, want_r, want_t, fh, 0.1, 0.3, 0.01)
    x = t(p.view(np.uint8))
    gpu_solver[1].add_smokeforce(x, r, tp, fh, 0.1, 0.3, 0.01)
    assert np.array_equal(x.cpu().numpy(), want.view(np.uint8))
    # an empty particle set is a no-op
    gpu_solver[1].add_smokeforce(t(np.zeros(0, np.uint8)), r, tp, fh, 0.1, 0.3, 0.01)
    assert len(want.view(PARTICLE_DTYPE)) == 200000


# ---- smoke tracers

def test_tracers_golden_and_oracle(gpu_solver, orc, tmp_path):
    """advect_tracers bit for bit against the reference's fixture; the
    on-disk file byte for byte; emit_tracers byte for byte against the oracle
    (same counter-based draws) and, in what the reference's rand() does not
    decide (kept tracers, their order, the count), against the fixture."""
    g = golden("tracers")
    s = gpu_solver[1]
    ni, nj, nk = (int(x) for x in g["dims"])
    h = float(g["h"])
    tr = t(g["tracers"])
    s.advect_tracers(ni, nj, nk, h, tr, t(g["u"]), t(g["v"]), t(g["w"]), t(g["phi"]), float(g["dt"]),
                     float(g["dens_decay"]))
    assert np.array_equal(bits(tr.cpu().numpy()), bits(g["advected"]))
    s.write_tracers(tr, float(g["lengths"][0]), tmp_path, 12)
    assert np.array_equal(np.fromfile(tmp_path / "Particle_data0012.bin", np.uint8), g["file_bytes"])
    e = s.emit_tracers(t(g["tracers"]), h, g["lengths"], (0.5, 0.2, 0.4), 0.1, 300, seed=1).cpu().numpy()
    assert len(e) == int(g["emit_count"])
    assert np.array_equal(bits(e[:-300]), bits(g["emit_kept"]))
    want = orc.emit_tracers(g["tracers"], h, g["lengths"], (0.5, 0.2, 0.4), 0.1, 300, seed=1)
    assert np.array_equal(bits(e), bits(want))


@pytest.mark.parametrize("n,count", [(0, 1000), (200000, 50000), (3, 0)])
def test_tracers_vs_oracle(gpu_solver, orc, n, count):
    rng = np.random.default_rng(53)
    ni, nj, nk = 32, 28, 24
    h = np.float32(1 / 32)
    lengths = (1.0, float(h * nj), float(h * nk))
    tr = np.concatenate([rng.uniform(-0.1, 1.1, (n, 3)), rng.uniform(0.0, 0.03, (n, 1))], 1).astype(np.float32)
    s = gpu_solver[1]
    got = s.emit_tracers(t(tr) if n else None, h, lengths, (0.5, 0.3, 0.4), 0.06, count, seed=4).cpu().numpy()
    want = orc.emit_tracers(tr, h, lengths, (0.5, 0.3, 0.4), 0.06, count, seed=4)
    assert np.array_equal(bits(got), bits(want))
    if len(want):
        phi = scenes.random_phi(ni, nj, nk, h, rng, n_spheres=3)
        u, v, w = scenes.random_velocity(ni, nj, nk, rng, scale=0.8)
        g = t(want)
        s.advect_tracers(ni, nj, nk, h, g, t(u), t(v), t(w), t(phi), 0.02, 0.5)
        assert np.array_equal(bits(g.cpu().numpy()), bits(orc.advect_tracers(ni, nj, nk, h, want, u, v, w, phi, 0.02,
                                                                              0.5)))
    # a capacity the result does not fit is refused
    if count:
        with pytest.raises(RuntimeError):
            s.emit_tracers(t(tr) if n else None, h, lengths, (0.5, 0.3, 0.4), 0.06, count, seed=4, capacity=count - 1)
