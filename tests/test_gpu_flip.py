"""GPU: the FLIP smoke step (advect_FLIP, P2G, emitter, projection, delta,
G2P with the 0.95 FLIP/PIC blend, reorder_FLIP) against the same step
composed from the oracle's functions, and a longer FP32 run's invariants."""
import numpy as np
import pytest

from vflip_b200.flip import FlipParams, FlipSim

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_flip_step_matches_oracle_composition(orc):
    from vflip_b200.solver import Solver

    n = 20
    prm = FlipParams(n=n, dt=0.02, source_radius=0.2)
    with Solver(precision=0) as s:
        sim = FlipSim(s, prm)
        p0 = sim.particles_host().copy()
        phi = sim.phi.cpu().numpy()
        src = sim.source_v.cpu().numpy()
        sim.step()
        got = sim.particles_host()
    h = np.float32(prm.h)
    zeros = [np.zeros(sh, np.float32) for sh in sim.shapes]
    p = orc.advect_flip(n, n, n, h, p0, *zeros, phi, prm.dt)
    u, _ = orc.p2g(n, n, n, h, p, 0)
    v, _ = orc.p2g(n, n, n, h, p, 1)
    w, _ = orc.p2g(n, n, n, h, p, 2)
    v[src] = prm.inflow
    out = orc.project(n, n, n, h, 0.0, phi, np.zeros((n, n, n), np.int8), *zeros, u, v, w)
    assert out["ok"]
    d = [out["u"] - u, out["v"] - v, out["w"] - w]
    p = orc.g2p(n, n, n, h, p, *d, out["u"], out["v"], out["w"], flip_ratio=prm.flip_ratio)
    want = orc.reorder_flip(n, n, n, h, p, out["u"], out["v"], out["w"], phi, seed=prm.seed)
    assert len(got) == len(want)
    assert np.allclose(got["pos"], want["pos"], rtol=0, atol=1e-6)
    assert np.allclose(got["vel"], want["vel"], rtol=1e-5, atol=1e-6)


def test_flip_sim_invariants():
    from vflip_b200.solver import Solver

    n = 32
    prm = FlipParams(n=n, dt=0.01)
    with Solver(precision=1) as s:
        sim = FlipSim(s, prm)
        n0 = sim.num_particles
        for _ in range(6):
            conv, st = sim.step()
            assert conv and st.residual <= 1e-6 * st.rhs_norm
        p = sim.particles_host()
        cells = s.particle_cells(n, n, n, prm.h, sim.particles).cpu().numpy()
    assert n0 < sim.num_particles and np.isfinite(p["vel"]).all()
    counts = np.bincount(cells[cells >= 0], minlength=n ** 3)
    assert counts.max() <= 9 and np.median(counts) == 8
    # the emitter pushes the smoke upward above the source
    above = p[(p["pos"][:, 1] > 0.15) & (p["pos"][:, 1] < 0.3) &
              (np.hypot(p["pos"][:, 0] - 0.5, p["pos"][:, 2] - 0.5) < 0.08)]
    assert len(above) > 0 and above["vel"][:, 1].mean() > 0.1


def test_flip_smoke_step_matches_oracle_composition(orc):
    """The density/temperature block (advect_field RK3 on the 2n grid,
    gen_heat, add_smokeforce) inside a FLIP step from an evolved state:
    density and temperature bit-exact, particles as above."""
    from vflip_b200.solver import Solver

    n = 20
    prm = FlipParams(n=n, dt=0.02, source_radius=0.2, smoke=True, smoke_radius=0.15, dens_decay=0.1,
                     temp_decay=0.2, alpha=0.1, beta=1.0)
    with Solver(precision=0) as s:
        sim = FlipSim(s, prm)
        sim.step()
        p1 = sim.particles_host().copy()
        vel1 = [x.cpu().numpy() for x in sim.vel]
        rho1, temp1 = sim.rho.cpu().numpy(), sim.temp.cpu().numpy()
        phi = sim.phi.cpu().numpy()
        src = sim.source_v.cpu().numpy()
        sim.step()
        got = sim.particles_host()
        got_rho, got_temp = sim.rho.cpu().numpy(), sim.temp.cpu().numpy()
    assert (rho1 == 1.0).any() and np.abs(vel1[1]).max() > 0
    h = np.float32(prm.h)
    fh = float(h) / 2
    p = orc.advect_flip(n, n, n, h, p1, *vel1, phi, prm.dt)
    rho = orc.advect_rk3(n, n, n, h, prm.dt, *vel1, rho1, fh)
    temp = orc.advect_rk3(n, n, n, h, prm.dt, *vel1, temp1, fh)
    rho, temp = orc.gen_heat(rho, temp, fh, prm.dt, prm.dens_decay, prm.temp_decay, prm.smoke_centre,
                             prm.smoke_radius, prm.smoke_dens, prm.smoke_heat)
    assert np.array_equal(got_rho.view(np.uint32), rho.view(np.uint32))
    assert np.array_equal(got_temp.view(np.uint32), temp.view(np.uint32))
    p = orc.add_smokeforce(p, rho, temp, fh, prm.alpha, prm.beta, prm.dt)
    u, _ = orc.p2g(n, n, n, h, p, 0)
    v, _ = orc.p2g(n, n, n, h, p, 1)
    w, _ = orc.p2g(n, n, n, h, p, 2)
    v[src] = prm.inflow
    zeros = [np.zeros(sh, np.float32) for sh in sim.shapes]
    out = orc.project(n, n, n, h, 0.0, phi, np.zeros((n, n, n), np.int8), *zeros, u, v, w)
    assert out["ok"]
    d = [out["u"] - u, out["v"] - v, out["w"] - w]
    p = orc.g2p(n, n, n, h, p, *d, out["u"], out["v"], out["w"], flip_ratio=prm.flip_ratio)
    want = orc.reorder_flip(n, n, n, h, p, out["u"], out["v"], out["w"], phi, seed=prm.seed + 1)
    assert len(got) == len(want)
    assert np.allclose(got["pos"], want["pos"], rtol=0, atol=1e-6)
    assert np.allclose(got["vel"], want["vel"], rtol=1e-5, atol=1e-5)


def test_flip_tracers(tmp_path):
    """Tracers ride along in the FLIP stepper: emitted in the source sphere
    every step, advected by the grid velocity, written in the reference's
    on-disk form."""
    from vflip_b200.solver import Solver

    with Solver(precision=1) as s:
        sim = FlipSim(s, FlipParams(n=32, dt=0.01, tracers_per_step=500))
        for _ in range(4):
            sim.step()
        tr = sim.tracers.cpu().numpy()
        sim.write_tracers(tmp_path, 4)
    # each emission first drops the tracers below 2h (the source sphere
    # reaches under it), then appends the new batch
    assert 1000 < len(tr) < 2000 and np.isfinite(tr).all()
    h = 1.0 / 32
    assert np.all(tr[:-500, 1] > 2 * h)
    assert tr[:-500, 1].mean() > tr[-500:, 1].mean()  # older tracers have risen with the flow
    rec = np.fromfile(tmp_path / "Particle_data0004.bin", np.float32).reshape(-1, 4)
    L = np.float32(1.0 / 32) * 32
    assert np.allclose(rec[:, 1], tr[:, 1] / L) and np.allclose(rec[:, 0], tr[:, 0] / L - 0.5)
