"""GPU: batched solves.  The graph-resident batch (one CUDA graph, each
system's PCG loop a device-side while node, systems as parallel branches)
gives the same iterates as solving the systems one after another: the same
iteration counts and bitwise-equal pressures, in every precision mode.  The
persistent batch (one cooperative kernel over all systems) converges to the
same tolerance with the graph's iteration counts (within one) and pressures
(to rounding), and every system of a config-2-style batch (random solid
spheres, uneven sides) matches the oracle's AMGPCGSolve."""
import numpy as np
import pytest

from vflip_b200 import scenes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_graph_batch_equals_per_system_loop(prec):
    from vflip_b200.solver import Solver

    # batched solves keep the PCG vectors in the working precision: the loop
    # is asked for the same (single solves default to FP64 vectors)
    with Solver(precision=prec, pcg_vectors=1) as s:
        systems = [scenes.batch_system(s, side, seed) for seed, side in enumerate((16, 24, 40, 32, 20))]
        ok_g, pg, sg = s.batched_solve(systems, 1e-6, 60, mode=0)
        ok_l, pl, sl = s.batched_solve(systems, 1e-6, 60, mode=1)
        assert ok_g and ok_l
        for a, b, x, y in zip(pg, pl, sg, sl):
            assert x.converged and x.iterations == y.iterations
            assert x.residual <= 1e-6 * x.rhs_norm
            assert torch.equal(a, b)


def test_graph_batch_edge_cases():
    from vflip_b200.solver import Solver

    with Solver(precision=1) as s:
        st, rhs = scenes.batch_system(s, 24, 3)
        zero = torch.zeros_like(rhs)
        ok, p, stats = s.batched_solve([(st, zero), (st, rhs)], 1e-6, 60, mode=0)
        assert ok and stats[0].iterations == 0 and float(p[0].abs().max()) == 0.0
        assert stats[1].iterations > 0
        # too few iterations: not converged, status 1, no error
        ok, _, stats = s.batched_solve([(st, rhs)], 1e-12, 2, mode=0)
        assert not ok and stats[0].iterations == 2 and not stats[0].converged
        ok, _, stats = s.batched_solve([], 1e-6, 10, mode=0)
        assert ok and stats == []


@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("chunk,ctas", [(0, 0), (1024, 1), (65536, 2)])
def test_persistent_batch_matches_graph(prec, chunk, ctas):
    from vflip_b200.solver import Solver

    with Solver(precision=prec, batch_chunk=chunk, batch_ctas_per_sm=ctas) as s:
        systems = [scenes.batch_system(s, side, seed) for seed, side in enumerate((16, 24, 40, 32, 20, 48, 17))]
        ok_g, pg, sg = s.batched_solve(systems, 1e-6, 60, mode=0)
        ok_p, pp, sp = s.batched_solve(systems, 1e-6, 60, mode=2)
        assert ok_g and ok_p
        for a, b, x, y in zip(pp, pg, sp, sg):
            assert x.converged and abs(x.iterations - y.iterations) <= 1
            assert x.residual <= 1e-6 * x.rhs_norm
            assert float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)) < 1e-4


def test_persistent_batch_edge_cases():
    from vflip_b200.solver import Solver

    with Solver(precision=1) as s:
        st, rhs = scenes.batch_system(s, 24, 3)
        zero = torch.zeros_like(rhs)
        ok, p, stats = s.batched_solve([(st, zero), (st, rhs)], 1e-6, 60, mode=2)
        assert ok and stats[0].iterations == 0 and float(p[0].abs().max()) == 0.0
        assert stats[1].iterations > 0 and stats[1].converged
        ok, _, stats = s.batched_solve([(st, rhs)], 1e-12, 2, mode=2)
        assert not ok and stats[0].iterations == 2 and not stats[0].converged
        ok, _, stats = s.batched_solve([], 1e-6, 10, mode=2)
        assert ok and stats == []
        # a NaN in one right-hand side makes that system's first rho NaN: it
        # stops at once (the reference returns false, 0 iterations); the other converges
        bad = rhs.clone()
        bad[5, 5, 5] = float("nan")
        ok, p, stats = s.batched_solve([(st, bad), (st, rhs)], 1e-6, 60, mode=2)
        assert not ok and not stats[0].converged and stats[0].iterations == 0
        assert stats[1].converged


def seven(st4):
    """(4, ...) device stencil (diag, +x, +y, +z) -> the oracle's (7, ...)
    slots diag, -x, +x, -y, +y, -z, +z (the -x coupling of a cell is the +x
    coupling of its left neighbour)."""
    d, xp, yp, zp = st4
    st = np.zeros((7,) + d.shape)
    st[0], st[2], st[4], st[6] = d, xp, yp, zp
    st[1][:, :, 1:] = xp[:, :, :-1]
    st[3][:, 1:, :] = yp[:, :-1, :]
    st[5][1:, :, :] = zp[:-1, :, :]
    return st


@pytest.mark.parametrize("mode,prec", [(0, 0), (0, 1), (2, 1), (2, 2)])
def test_batch_systems_match_the_oracle(orc, mode, prec):
    """Config-2-style systems (random spheres of radius 0.05-0.25 of the side,
    rhs the divergence of a smoothed Gaussian velocity), uneven sides: each
    batched pressure against the oracle's AMGPCGSolve of the same system
    (FP64 with the reference's hierarchy).  FP64 graph mode reproduces it to
    1e-9 with the same iteration count; FP32 and mixed, with their own
    hierarchy and stopping point, to 1e-4 relative L2 (the bar of a single
    FP32 solve against the reference)."""
    from vflip_b200.solver import Solver

    with Solver(precision=prec) as s:
        systems, sides = scenes.batch_workload(s, count=6, seed=5, sides=(16, 24, 32, 40))
        ok, ps, stats = s.batched_solve(systems, 1e-6, 100, mode=mode)
        assert ok
        for (st, rhs), p, x in zip(systems, ps, stats):
            want, wok, _, wit = orc.amgpcg(seven(st.cpu().numpy()), rhs.cpu().numpy())
            assert wok and x.converged
            err = np.linalg.norm(p.cpu().numpy() - want) / np.linalg.norm(want)
            assert err < (1e-9 if prec == 0 else 1e-4), (rhs.shape, err)
            if prec == 0:
                assert x.iterations == wit
