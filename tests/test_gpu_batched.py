"""GPU: batched solves.  The graph-resident batch (one CUDA graph, each
system's PCG loop a device-side while node, systems as parallel branches)
gives the same iterates as solving the systems one after another: the same
iteration counts and bitwise-equal pressures, in every precision mode."""
import pytest

from vflip_b200 import scenes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_graph_batch_equals_per_system_loop(prec):
    from vflip_b200.solver import Solver

    with Solver(precision=prec) as s:
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
