"""Host-side pieces of bench.py that need no GPU."""
import numpy as np

import bench
import oracle
from vflip_b200 import scenes


def test_csr_of_stencil_matches_the_full_pattern_without_zero_couplings():
    """bench.csr_of_stencil (the CSR the drop-in timing hands over) is the
    oracle's full 7-point CSR with the zero off-diagonal entries left out,
    as SmokeSolver3D::pcg_projection leaves them out for solid neighbours."""
    pr = scenes.projection_problem(13, 11, 9, seed=3, inflow=True, solid_velocity=True)
    orc = oracle.oracle()
    st7 = orc.project(**pr)["stencil"]
    st4 = np.stack([st7[0], st7[2], st7[4], st7[6]])
    rs, ci, v = bench.csr_of_stencil(st4)
    frs, fci, fv = oracle.stencil_to_csr(st7)
    n = len(rs) - 1
    assert n == 13 * 11 * 9
    for r in range(n):
        full = [(c, x) for c, x in zip(fci[frs[r]:frs[r + 1]], fv[frs[r]:frs[r + 1]]) if x != 0 or c == r]
        got = list(zip(ci[rs[r]:rs[r + 1]], v[rs[r]:rs[r + 1]]))
        assert got == full, r
    rows = np.repeat(np.arange(n), np.diff(rs.astype(np.int64)))
    assert np.all((v != 0) | (ci == rows))
