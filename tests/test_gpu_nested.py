"""GPU parity of the main grid's routines with its nested subdomain active
(the blended get_velocity, the subdomain's solid phi and normal, the halo
selection and the subdomain's tracer seeding): bit-exact against the
reference's fixture and against the oracle, seeded draws included (both use
the same counter-based generator)."""
import hashlib

import numpy as np
import pytest

from conftest import nested_from_golden
from vflip_b200 import scenes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def device_sub(s, sub):
    return s.subdomain(sub["dims"], sub["h"], sub["bmin"], t(sub["u"]), t(sub["v"]), t(sub["w"]), t(sub["phi"]))


def test_nested_golden(gpu_solver):
    s = gpu_solver[1]
    g, sub = nested_from_golden()
    ni, nj, nk = (int(x) for x in g["dims"])
    h = float(g["h"])
    u, v, w, phi = t(g["u"]), t(g["v"]), t(g["w"]), t(g["phi"])
    ds = device_sub(s, sub)
    p = t(g["particles"])
    s.advect_flip_nested(ni, nj, nk, h, p, u, v, w, phi, 0.01, ds)
    assert np.array_equal(p.cpu().numpy(), g["advect"])
    r = s.reorder_flip_nested(ni, nj, nk, h, t(g["jittered"]), u, v, w, phi, ds)
    assert r.numel() // 40 == int(g["reorder_count"])
    assert hashlib.sha256(r.cpu().numpy().tobytes()).hexdigest() == str(g["reorder_sha256"])
    halo = s.halo_select(t(g["particles"]), h, ds)
    assert np.array_equal(halo.cpu().numpy(), g["halo"])
    tr = t(g["tracers"])
    s.advect_tracers_nested(ni, nj, nk, h, tr, u, v, w, phi, 0.01, 0.1, ds)
    assert np.array_equal(tr.cpu().numpy().view(np.uint32), g["tracers_advected"].view(np.uint32))
    lengths = np.array([ni, nj, nk], np.float32) * np.float32(h)
    e = s.emit_tracers_nested(t(g["tracers"]), h, lengths, (0.3, 0.15, 0.25), 0.06, 400, (ni, nj, nk), phi, ds,
                              seed=5).cpu().numpy()
    kept = g["emit_kept"]
    assert np.array_equal(e[:len(kept)].view(np.uint32), kept.view(np.uint32))
    n = int(g["emit_count"]) - len(kept) - 400
    assert abs(len(e) - len(kept) - 400 - n) <= 5 * np.sqrt(2 * n) + 5


@pytest.mark.parametrize("seed,dims,lo,cells", [(11, (18, 16, 14), (5, 4, 3), (9, 8, 7)),
                                                (12, (48, 40, 36), (12, 10, 9), (24, 20, 18))])
def test_nested_vs_oracle(gpu_solver, orc, seed, dims, lo, cells):
    s = gpu_solver[1]
    sc = scenes.nested_scene(seed=seed, dims=dims, lo=lo, cells=cells)
    ni, nj, nk = sc["dims"]
    h, sub, rng = sc["h"], sc["sub"], sc["rng"]
    un, vn, wn, phin = sc["u"], sc["v"], sc["w"], sc["phi"]
    u, v, w, phi = t(un), t(vn), t(wn), t(phin)
    ds = device_sub(s, sub)
    p = scenes.random_particles(ni, nj, nk, h, 8 * ni * nj * nk // 3, rng, margin=2.0)
    # advect_FLIP through the blend
    x = t(p.view(np.uint8))
    s.advect_flip_nested(ni, nj, nk, h, x, u, v, w, phi, 0.02, ds)
    want = orc.advect_flip_nested(ni, nj, nk, h, p, un, vn, wn, phin, 0.02, sub)
    assert np.array_equal(x.cpu().numpy(), want.view(np.uint8))
    # halo selection
    assert np.array_equal(s.halo_select(t(p.view(np.uint8)), h, ds).cpu().numpy(),
                          orc.halo_select(p, h, sub).view(np.uint8))
    # reorder with seeding: same counter-based draws, nested solid filter
    r = s.reorder_flip_nested(ni, nj, nk, h, t(p.view(np.uint8)), u, v, w, phi, ds, seed=9)
    want = orc.reorder_flip_nested(ni, nj, nk, h, p, un, vn, wn, phin, sub, seed=9)
    assert np.array_equal(r.cpu().numpy(), want.view(np.uint8))
    # tracers: advection and emission with the subdomain's seeding
    tr = np.concatenate([p["pos"], rng.uniform(0.0, 1.0, (len(p), 1)).astype(np.float32)], 1)
    y = t(tr)
    s.advect_tracers_nested(ni, nj, nk, h, y, u, v, w, phi, 0.02, 0.2, ds)
    want = orc.advect_tracers_nested(ni, nj, nk, h, tr, un, vn, wn, phin, 0.02, 0.2, sub)
    assert np.array_equal(y.cpu().numpy().view(np.uint32), want.view(np.uint32))
    lengths = np.array([ni, nj, nk], np.float32) * h
    e = s.emit_tracers_nested(t(tr), h, lengths, (0.4, 0.2, 0.3), 0.05, 700, (ni, nj, nk), phi, ds, seed=3)
    want = orc.emit_tracers_nested(tr, h, lengths, (0.4, 0.2, 0.3), 0.05, 700, (ni, nj, nk), phin, sub, seed=3)
    plain = orc.emit_tracers(tr, h, lengths, (0.4, 0.2, 0.3), 0.05, 700, seed=3)
    assert len(want) > len(plain) and np.array_equal(want[:len(plain)], plain)  # seeds follow the plain emission
    assert np.array_equal(e.cpu().numpy().view(np.uint32), want.view(np.uint32))


def test_nested_argument_errors(gpu_solver):
    from vflip_b200._lib import VflipError

    s = gpu_solver[1]
    sc = scenes.nested_scene(seed=1)
    ni, nj, nk = sc["dims"]
    sub = dict(sc["sub"])
    bad = device_sub(s, dict(sub, h=np.float32(0.0)))
    p = t(scenes.random_particles(ni, nj, nk, sc["h"], 100, sc["rng"]).view(np.uint8))
    with pytest.raises(VflipError):
        s.halo_select(p, sc["h"], bad)
    with pytest.raises(VflipError):
        s.advect_flip_nested(ni, nj, nk, sc["h"], p, t(sc["u"]), t(sc["v"]), t(sc["w"]), t(sc["phi"]), 0.01, bad)
    # capacity short: the count is still reported
    ds = device_sub(s, sub)
    with pytest.raises(VflipError):
        s.halo_select(t(scenes.jittered_particles(ni, nj, nk, sc["h"], 8, sc["rng"]).view(np.uint8)), sc["h"], ds,
                      capacity=1)


def _host(x):
    import oracle

    return x.cpu().numpy().view(oracle.PARTICLE_DTYPE).copy()


def test_nested_step_matches_oracle_composition(orc):
    """The second coupled step of a small plume (FP64 context) against the
    same step composed from the oracle's functions in time_step's order."""
    from vflip_b200.flip import NestedFlipSim, NestedParams
    from vflip_b200.solver import Solver

    n = 24
    prm = NestedParams(n=n, dt=0.02, source_radius=0.2, obstacle_radius=0.0, seed=4)
    with Solver(precision=0) as s:
        sim = NestedFlipSim(s, prm)
        sim.step()
        p0, sp0 = sim.particles_host().copy(), _host(sim.sub_particles)
        vel = [x.cpu().numpy() for x in sim.vel]
        svel = [x.cpu().numpy() for x in sim.sub_vel]
        phi, sphi, src = sim.phi.cpu().numpy(), sim.sphi.cpu().numpy(), sim.source_v.cpu().numpy()
        conv, _, sstats = sim.step()
        assert conv and sstats.iterations > 0
        got, sgot = sim.particles_host(), _host(sim.sub_particles)
        gvel = [x.cpu().numpy() for x in sim.vel]
    h, sh, bmin, seed = np.float32(prm.h), sim.sh, sim.bmin, prm.seed + 1
    sni, snj, snk = sim.sdims
    sub = dict(dims=sim.sdims, h=sh, bmin=bmin, u=svel[0], v=svel[1], w=svel[2], phi=sphi)
    zeros = [np.zeros(a.shape, np.float32) for a in vel]
    p = orc.advect_flip_nested(n, n, n, h, np.concatenate([p0, sp0]), *vel, phi, prm.dt, sub)
    u, v, w = (orc.p2g(n, n, n, h, p, c)[0] for c in range(3))
    v[src] = prm.inflow
    out = orc.project(n, n, n, h, 0.0, phi, np.zeros((n, n, n), np.int8), *zeros, u, v, w)
    assert out["ok"]
    p = orc.g2p(n, n, n, h, p, out["u"] - u, out["v"] - v, out["w"] - w, out["u"], out["v"], out["w"],
                flip_ratio=prm.flip_ratio)
    q = orc.halo_select(p, h, sub)
    su, sv, sw = (orc.sub_p2g(sni, snj, snk, sh, bmin, q, c)[0] for c in range(3))
    szeros = [np.zeros(a.shape, np.float32) for a in (su, sv, sw)]
    so = orc.project_subdomain(sni, snj, snk, sh, 1.0, sphi, *szeros, su, sv, sw)
    assert so["ok"]
    q = orc.sub_g2p(sni, snj, snk, sh, bmin, q, so["u"] - su, so["v"] - sv, so["w"] - sw)
    q = orc.sub_reorder_flip(sni, snj, snk, sh, bmin, q, so["u"], so["v"], so["w"], sphi, seed=seed ^ 0x5EED)
    sub2 = dict(sub, u=so["u"], v=so["v"], w=so["w"])
    want = orc.reorder_flip_nested(n, n, n, h, p, out["u"], out["v"], out["w"], phi, sub2, seed=seed)
    assert len(got) == len(want) and len(sgot) == len(q)
    for a, b in ((got, want), (sgot, q)):
        assert np.array_equal(a["pos"], b["pos"]) or np.allclose(a["pos"], b["pos"], rtol=0, atol=1e-6)
        assert np.allclose(a["vel"], b["vel"], rtol=1e-5, atol=1e-6)
    assert np.allclose(gvel[1], out["v"], rtol=1e-5, atol=1e-6)


def test_nested_sim_invariants_mixed():
    """A few coupled steps in the mixed-precision context: both solves
    converge, the subdomain keeps 8 particles per open interior cell, and
    its particles ride the main pass (main count includes them)."""
    from vflip_b200.flip import NestedFlipSim, NestedParams
    from vflip_b200.solver import Solver

    prm = NestedParams(n=32, dt=0.01, obstacle_radius=0.1, tracers_per_step=300)
    with Solver(precision=2) as s:
        sim = NestedFlipSim(s, prm)
        sni, snj, snk = sim.sdims
        for _ in range(4):
            conv, stats, sstats = sim.step()
            assert conv
            assert 0 < sim.num_sub_particles <= 9 * (sni - 2) * (snj - 2) * (snk - 2)
            sp = _host(sim.sub_particles)
            assert np.isfinite(sp["vel"]).all() and np.isfinite(sim.particles_host()["vel"]).all()
        assert sim.tracers.shape[0] > 300
        assert float(sim.sub_vel[1].abs().max()) > 0.0


def test_nested_empty_inputs(gpu_solver):
    """No particles and no tracers: every nested call returns cleanly and
    emission seeds only the subdomain's cells."""
    s = gpu_solver[1]
    sc = scenes.nested_scene(seed=2)
    ni, nj, nk = sc["dims"]
    h = sc["h"]
    u, v, w, phi = t(sc["u"]), t(sc["v"]), t(sc["w"]), t(sc["phi"])
    ds = device_sub(s, sc["sub"])
    empty = torch.zeros(0, dtype=torch.uint8, device=DEV)
    assert s.halo_select(empty, h, ds).numel() == 0
    s.advect_flip_nested(ni, nj, nk, h, empty, u, v, w, phi, 0.01, ds)
    r = s.reorder_flip_nested(ni, nj, nk, h, empty, u, v, w, phi, ds, seed=1)
    assert r.numel() > 0 and r.numel() % 40 == 0  # every open cell seeded with 8
    lengths = np.array([ni, nj, nk], np.float32) * h
    e = s.emit_tracers_nested(None, h, lengths, (0.3, 0.2, 0.3), 0.05, 0, (ni, nj, nk), phi, ds, seed=4)
    assert e.shape[1] == 4 and (e[:, 3] == 1).all()
    tr = torch.zeros((0, 4), dtype=torch.float32, device=DEV)
    s.advect_tracers_nested(ni, nj, nk, h, tr, u, v, w, phi, 0.01, 0.1, ds)
