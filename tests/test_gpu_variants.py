"""Kernel variants that must agree with the kernels they replace:
  * the tiled RK2 advection (velocity grids staged in shared memory) gives
    the per-node gather kernel's bits, in FP64 (the reference's arithmetic)
    and FP32 contexts, for slow flow (every sample inside the staged halo)
    and fast flow (samples beyond it take the global sampler);
  * the one-launch u, v, w advection gives the three single launches' bits;
  * the plane-marching PCG SpMV gives the column kernel's iterations and,
    up to the grouping of its s.q partial sums, its solution."""
import numpy as np
import pytest

from vflip_b200 import scenes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


@pytest.fixture(scope="module")
def pairs():
    from vflip_b200.solver import Solver

    s = {(p, k): Solver(precision=p, advect_kernel=k) for p in (0, 1) for k in (0, 1)}
    yield s
    for v in s.values():
        v.close()


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
@pytest.mark.parametrize("amp,dt", [(0.3, 0.02), (4.0, 0.05)])
def test_tiled_advection_matches_gather_kernel(pairs, prec, amp, dt):
    ni, nj, nk = 40, 36, 33
    h = np.float32(1.0 / 40)
    u, v, w = smooth_velocity(ni, nj, nk, amp, seed=3)
    rng = np.random.default_rng(4)
    U, V, W = t(u), t(v), t(w)
    offs = {"u": (0.5, 0, 0), "v": (0, 0.5, 0), "w": (0, 0, 0.5)}
    for name, f in zip("uvw", (U, V, W)):
        # the field is a velocity grid (self-advection) and, separately, an unrelated field on that grid
        other = t(rng.standard_normal(f.shape).astype(np.float32))
        for fld in (f, other):
            a = pairs[(prec, 0)].advect_rk2_linear(ni, nj, nk, h, dt, U, V, W, fld, offs[name])
            b = pairs[(prec, 1)].advect_rk2_linear(ni, nj, nk, h, dt, U, V, W, fld, offs[name])
            assert torch.equal(a, b), name
    r = t(rng.standard_normal((nk, nj, ni)).astype(np.float32))
    q = t(rng.standard_normal((nk, nj, ni)).astype(np.float32))
    a = pairs[(prec, 0)].advect_rk2_linear2(ni, nj, nk, h, dt, U, V, W, r, q, (0, 0, 0))
    b = pairs[(prec, 1)].advect_rk2_linear2(ni, nj, nk, h, dt, U, V, W, r, q, (0, 0, 0))
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("dims", [(40, 36, 33), (64, 32, 16), (1, 9, 70)])
def test_velocity_advection_one_launch(pairs, prec, dims):
    ni, nj, nk = dims
    h = np.float32(1.0 / max(dims))
    u, v, w = smooth_velocity(ni, nj, nk, 2.0, seed=5)
    U, V, W = t(u), t(v), t(w)
    s = pairs[(prec, 0)]
    got = s.advect_velocity_rk2_linear(ni, nj, nk, h, 0.03, U, V, W)
    for name, f, o, g in zip("uvw", (U, V, W), ((0.5, 0, 0), (0, 0.5, 0), (0, 0, 0.5)), got):
        want = pairs[(prec, 1)].advect_rk2_linear(ni, nj, nk, h, 0.03, U, V, W, f, o)
        assert torch.equal(g, want), name
    # the gather form of the one-call entry point too
    got1 = pairs[(prec, 1)].advect_velocity_rk2_linear(ni, nj, nk, h, 0.03, U, V, W)
    for a, b in zip(got, got1):
        assert torch.equal(a, b)


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
