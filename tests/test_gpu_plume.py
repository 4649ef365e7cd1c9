"""GPU: whole plume steps (advection + sources + projection) against the
oracle's step, config-0 scene (64^3, dt = 0.02, 20 steps, no obstacle) and a
shorter obstacle run."""
import numpy as np
import pytest

from vflip_b200.plume import PlumeParams, PlumeSim, nodal_phi

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.parametrize("prec,n,steps,obstacle,tol", [(0, 64, 20, False, 1e-5), (1, 64, 20, False, 1e-3),
                                                       (0, 40, 5, True, 1e-5)])
def test_plume_matches_oracle(gpu_solver, orc, prec, n, steps, obstacle, tol):
    p = PlumeParams(n=n, dt=0.02, obstacle=obstacle)
    sim = PlumeSim(gpu_solver[prec], p)
    phi = nodal_phi(p)
    state = {k: np.zeros(sim.shapes[k], np.float32) for k in sim.FIELDS}
    for s in range(steps):
        ok, it, res = orc.smoke_step(n, p.h, p.dt, phi, state)
        conv, stats = sim.step()
        assert conv and ok
        if prec == 0:
            assert stats.iterations == it
    for k in sim.FIELDS:
        assert rel(sim.f[k].cpu().numpy(), state[k]) < tol, k
    # the projected field is (discretely) divergence free where the solve acts
    assert float(np.abs(state["v"]).max()) > 0.05


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_projection_removes_divergence(gpu_solver, prec):
    """After the projection the weighted divergence is the solve's residual:
    at a 1e-6 inf-norm tolerance it drops by orders of magnitude."""
    p = PlumeParams(n=48, dt=0.02, obstacle=True)
    sim = PlumeSim(gpu_solver[prec], p)
    for _ in range(3):
        sim.step()
    sim.advect_and_force()
    before = float(sim.divergence(sim.f["u"], sim.f["v"], sim.f["w"]).abs().max())
    conv, _, st = sim.project()
    after = float(sim.divergence(sim.f["u"], sim.f["v"], sim.f["w"]).abs().max())
    assert conv and before > 0.1
    assert after < 1e-3 * before, (before, after)


def test_step_host_matches_device_steps(gpu_solver):
    """Steps on host-resident state (the end-to-end path: fields copied in and
    out every step on three copy streams) give the device-resident steps'
    fields bit for bit."""
    p = PlumeParams(n=48, dt=0.02, obstacle=True)
    a = PlumeSim(gpu_solver[1], p)
    b = PlumeSim(gpu_solver[1], p)
    host = {k: torch.zeros(a.shapes[k], dtype=torch.float32, pin_memory=True) for k in a.FIELDS}
    for _ in range(4):
        a.step()
        b.step_host(host)
    b.host_join()
    torch.cuda.synchronize()
    for k in a.FIELDS:
        assert np.array_equal(a.f[k].cpu().numpy(), host[k].numpy()), k
    assert float(host["rho"].abs().max()) > 0 and float(host["v"].abs().max()) > 0
