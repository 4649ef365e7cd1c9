"""GPU: the learned-preconditioned projection.  Capture mode is the plain
solve (identical results); the learned solve converges to the same
tolerance whatever the network outputs (random, or non-finite), and the
answer agrees with the plain solve's."""
import numpy as np
import pytest

from vflip_b200.learned import CAPTURE, NO_VB, SOLVE, LearnedPreconditioner, UNet
from vflip_b200.plume import PlumeParams, PlumeSim

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _state(prec, n=40, steps=4):
    from vflip_b200.solver import Solver

    s = Solver(precision=prec)
    sim = PlumeSim(s, PlumeParams(n=n, dt=0.02))
    for _ in range(steps):
        sim.step()
    sim.advect_and_force()
    return s, sim


def _rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


@pytest.mark.parametrize("prec", [0, 1])
def test_capture_is_the_plain_solve(prec):
    s, sim = _state(prec)
    u0 = {k: sim.f[k].clone() for k in ("u", "v", "w")}
    conv, p_plain, st, = sim.project()[:3]
    p_plain = p_plain.clone()
    u_plain = {k: sim.f[k].clone() for k in ("u", "v", "w")}
    for k in u0:
        sim.f[k].copy_(u0[k])
    n = sim.p.n
    X, Y, Z = s.learned_grid(n, n, n, 1)
    assert (X, Y, Z) == (24, 24, 24)
    smp = (torch.empty((Z, Y, X, 2), device="cuda"), torch.empty((Z, Y, X, 2), device="cuda"),
           torch.empty((Z, Y, X), device="cuda"))
    conv2, p2, st2, _ = sim.project_learned(None, CAPTURE, 1, sample=smp)
    assert conv and conv2 and st2.iterations == st.iterations
    assert torch.equal(p2, p_plain)
    for k in u0:
        assert torch.equal(sim.f[k], u_plain[k])
    in2, t2, w = (x.cpu().numpy() for x in smp)
    assert np.array_equal(in2[..., 1], w) and w.min() >= 0 and w.max() <= 1
    assert np.abs(in2[..., 0]).max() == pytest.approx(1.0)
    # targets are R p and R (p - x1) scaled like the features: channel 0
    # equals the block average of the pressure times the feature scale
    p = p_plain.cpu().numpy()
    pad = np.zeros((Z * 2, Y * 2, X * 2))
    pad[:n, :n, :n] = p
    avg = pad.reshape(Z, 2, Y, 2, X, 2).mean(axis=(1, 3, 5))
    m = np.abs(avg) > 1e-3 * np.abs(avg).max()
    ratio = t2[..., 0][m] / avg[m]
    assert np.allclose(ratio, ratio.mean(), rtol=1e-4)
    assert np.isfinite(t2).all()


@pytest.mark.parametrize("prec,mode", [(0, SOLVE), (1, SOLVE), (1, SOLVE | NO_VB), (2, SOLVE)])
def test_learned_solve_converges_to_plain_answer(prec, mode):
    s, sim = _state(prec)
    u0 = {k: sim.f[k].clone() for k in ("u", "v", "w")}
    _, p_plain, st = sim.project()
    p_plain = p_plain.clone()
    for k in u0:
        sim.f[k].copy_(u0[k])
    with UNet(seed=7) as net:
        conv, p, st2, ls = sim.project_learned(net, mode, 1)
    assert conv and st2.converged
    assert st2.residual <= 1e-6 * st2.rhs_norm
    assert _rel(p, p_plain) < (1e-5 if prec == 0 else 2e-3)
    assert ls.net_ms > 0


def test_learned_solve_survives_non_finite_network():
    s, sim = _state(1)
    with UNet(seed=7) as net:
        p = net.get_params()
        p[:] = np.nan
        net.set_params(p)
        conv, _, st, ls = sim.project_learned(net, SOLVE, 1)
    assert conv and st.residual <= 1e-6 * st.rhs_norm
    assert ls.subspace <= 1 and ls.gamma[1] == 0 and ls.gamma[2] == 0


def test_learned_mode_arguments():
    from vflip_b200._lib import VflipError

    s, sim = _state(1, n=24, steps=1)
    with pytest.raises(VflipError):
        sim.project_learned(None, SOLVE, 1)
    with pytest.raises(VflipError):
        sim.project_learned(None, CAPTURE, 1)
    with pytest.raises(VflipError):
        sim.project_learned(None, CAPTURE | SOLVE, 1)


def test_previous_pressure_without_network():
    # ablation mode: no network, the incoming (previous) pressure joins V(b)
    s, sim = _state(1)
    from vflip_b200.learned import PREV, NO_NET

    conv, _, st, ls = sim.project_learned(None, SOLVE | PREV | NO_NET, 1)
    assert conv and st.residual <= 1e-6 * st.rhs_norm
    assert ls.gamma[1] == 0 and ls.gamma[2] == 0 and ls.net_ms == 0


def test_training_improves_the_warm_start():
    """What the trained network gains over the untrained one: on held-out
    steps its warm start (Ritz step without V(b)) leaves a much smaller
    residual, and the solve needs no more V-cycles."""
    from vflip_b200.solver import Solver

    s = Solver(precision=1)
    sim = PlumeSim(s, PlumeParams(n=48, dt=0.01))
    for _ in range(6):
        sim.step()
    pre = LearnedPreconditioner(s, level=0, seed=1, use_vb=False, sweeps=2)
    for _ in range(24):
        sim.step(pre)
    with UNet(seed=1) as fresh:
        untrained = LearnedPreconditioner(s, level=0, net=fresh, use_vb=False, sweeps=2)
        untrained.capturing = False
        pre.train(epochs=20, lr=1e-3)
        r_tr, r_un, vc_tr, vc_un = [], [], [], []
        for _ in range(3):
            sim.advect_and_force()
            u0 = {k: sim.f[k].clone() for k in ("u", "v", "w")}
            p0 = sim.pressure.clone()
            for which, rr, vv in ((untrained, r_un, vc_un), (pre, r_tr, vc_tr)):
                for k in u0:
                    sim.f[k].copy_(u0[k])
                sim.pressure.copy_(p0)
                conv, st = which.project(sim)
                assert conv
                rr.append(which.last.init_residual / st.rhs_norm)
                vv.append(st.vcycles)
    assert np.mean(r_tr) < 0.6 * np.mean(r_un), (r_tr, r_un)
    assert np.mean(vc_tr) <= np.mean(vc_un), (vc_tr, vc_un)


# ---- the warm-start correction (VFLIP_LEARNED_RESID)

@pytest.mark.parametrize("prec", [0, 1])
def test_resid_capture_is_the_plain_solve(prec):
    """Capture in residual mode solves like the plain projection (same bits)
    and records target = R^L (p_new - p_prev) scaled like the features."""
    from vflip_b200.learned import RESID

    s, sim = _state(prec)
    p_prev = sim.pressure.clone()
    u0 = {k: sim.f[k].clone() for k in ("u", "v", "w")}
    conv, p_plain, st = sim.project()
    p_plain = p_plain.clone()
    for k in u0:
        sim.f[k].copy_(u0[k])
    sim.pressure.copy_(p_prev)
    n = sim.p.n
    X, Y, Z = s.learned_grid(n, n, n, 1)
    smp = (torch.empty((Z, Y, X, 2), device="cuda"), torch.empty((Z, Y, X, 2), device="cuda"),
           torch.empty((Z, Y, X), device="cuda"))
    conv2, p2, st2, _ = sim.project_learned(None, CAPTURE | RESID, 1, sample=smp)
    assert conv and conv2 and st2.iterations == st.iterations
    assert torch.equal(p2, p_plain)
    in2, t2, w = (x.cpu().numpy() for x in smp)
    assert np.abs(in2[..., 0]).max() == pytest.approx(1.0)
    d = (p_plain - p_prev).cpu().numpy()
    pad = np.zeros((Z * 2, Y * 2, X * 2))
    pad[:n, :n, :n] = d
    avg = pad.reshape(Z, 2, Y, 2, X, 2).mean(axis=(1, 3, 5))
    m = np.abs(avg) > 1e-3 * np.abs(avg).max()
    ratio = t2[..., 0][m] / avg[m]
    assert np.allclose(ratio, ratio.mean(), rtol=1e-4)
    assert np.array_equal(t2[..., 0], t2[..., 1])


@pytest.mark.parametrize("prec,net_on,sweeps", [(1, False, 0), (1, True, 2), (2, True, 2), (0, True, 0)])
def test_resid_solve_converges_to_plain_answer(prec, net_on, sweeps):
    """Whatever the network says (here an untrained one), the residual-mode
    solve reaches the plain solve's tolerance and, up to where two solves
    from different starting points stop inside it, its answer (both with
    FP64 PCG vectors)."""
    from vflip_b200.learned import NO_NET, RESID, SWEEPS

    s, sim = _state(prec)
    p_prev = sim.pressure.clone()
    u0 = {k: sim.f[k].clone() for k in ("u", "v", "w")}
    _, p_plain, st = sim.project()
    p_plain = p_plain.clone()
    for k in u0:
        sim.f[k].copy_(u0[k])
    sim.pressure.copy_(p_prev)
    with UNet(seed=7) as net:
        mode = SOLVE | RESID | SWEEPS(sweeps) | (0 if net_on else NO_NET)
        conv, p, st2, ls = sim.project_learned(net if net_on else None, mode, 1)
    assert conv and st2.converged
    assert st2.residual <= 1e-6 * st2.rhs_norm
    assert _rel(p, p_plain) < 1e-4
    assert (ls.net_ms > 0) == net_on
    if not net_on:
        assert ls.gamma[1] == 0


def test_resid_mode_needs_fp64_vectors():
    from vflip_b200._lib import VflipError
    from vflip_b200.learned import NO_NET, RESID
    from vflip_b200.solver import Solver

    s = Solver(precision=1, pcg_vectors=1)
    sim = PlumeSim(s, PlumeParams(n=24, dt=0.02))
    sim.advect_and_force()
    with pytest.raises(VflipError):
        sim.project_learned(None, SOLVE | RESID | NO_NET, 1)


@pytest.mark.parametrize("prec,net_on", [(1, False), (1, True), (2, True)])
def test_resid_solve_device_loop_equals_host_loop(prec, net_on):
    """The warm-started PCG runs as the device-resident loop (a CUDA graph
    with a conditional while node); the host loop (pcg_loop=1) gives the
    same bits, iterations and Ritz coefficients.  Plain and warm-started
    solves alternating on one context keep their own graphs."""
    from vflip_b200.learned import NO_NET, RESID, SWEEPS
    from vflip_b200.solver import Solver

    out = []
    for loop in (0, 1):
        s = Solver(precision=prec, pcg_loop=loop)
        sim = PlumeSim(s, PlumeParams(n=40, dt=0.02))
        for _ in range(4):
            sim.step()
        sim.advect_and_force()
        p_prev = sim.pressure.clone()
        u0 = {k: sim.f[k].clone() for k in ("u", "v", "w")}
        res = []
        with UNet(seed=7) as net:
            mode = SOLVE | RESID | SWEEPS(2) | (0 if net_on else NO_NET)
            for rep in range(2):
                for k in u0:
                    sim.f[k].copy_(u0[k])
                sim.pressure.copy_(p_prev)
                _, p_plain, st_plain = sim.project()
                p_plain = p_plain.clone()
                for k in u0:
                    sim.f[k].copy_(u0[k])
                sim.pressure.copy_(p_prev)
                conv, p, st, ls = sim.project_learned(net if net_on else None, mode, 1)
                res.append((p.clone(), st.iterations, tuple(ls.gamma[:2]), p_plain, st_plain.iterations))
        out.append(res)
        s.close()
    for (pa, ia, ga, qa, ja), (pb, ib, gb, qb, jb) in zip(*out):
        assert torch.equal(pa, pb) and ia == ib and ga == gb
        assert torch.equal(qa, qb) and ja == jb
    assert torch.equal(out[0][0][0], out[0][1][0])
