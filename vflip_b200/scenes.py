"""Seeded synthetic scenes in this library's linear layout (i fastest).

All arrays are numpy, shaped (z, y, x).  For an ni x nj x nk cell grid of
spacing h (cell (i,j,k) centred at (i,j,k)*h, as the reference places it):
  u faces (nk, nj, ni+1) at world ((i-1/2)h, jh, kh)
  v faces (nk, nj+1, ni) at world (ih, (j-1/2)h, kh)
  w faces (nk+1, nj, ni) at world (ih, jh, (k-1/2)h)
  nodal solid phi (nk+1, nj+1, ni+1) at world ((i-1/2)h, (j-1/2)h, (k-1/2)h)
matching SmokeSolver3D::init and set_boundary_phi (Smoke_solver3D.h:299-328,
Smoke_solver3D.cpp:864).
"""
import numpy as np

from .particles import PARTICLE_DTYPE


def nodal_coords(ni, nj, nk, h):
    z, y, x = np.meshgrid(np.arange(nk + 1), np.arange(nj + 1), np.arange(ni + 1), indexing="ij")
    return (x - 0.5) * h, (y - 0.5) * h, (z - 0.5) * h


def sphere_phi(ni, nj, nk, h, centre, radius):
    """Solid sphere signed distance at the nodes: negative inside the solid."""
    x, y, z = nodal_coords(ni, nj, nk, h)
    d = np.sqrt((x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2)
    return (d - radius).astype(np.float32)


def box_walls_phi(ni, nj, nk, h, open_top=True):
    """Distance to solid walls one cell thick on the five faces (all six if
    open_top is False); positive in the fluid, negative in the walls."""
    x, y, z = nodal_coords(ni, nj, nk, h)
    lx, ly, lz = ni * h, nj * h, nk * h
    walls = [x - h, (lx - 2 * h) - x, y - h, z - h, (lz - 2 * h) - z]
    if not open_top:
        walls.append((ly - 2 * h) - y)
    return np.minimum.reduce(walls).astype(np.float32)


def random_phi(ni, nj, nk, h, rng, n_spheres=3):
    """Union of a few random solid spheres plus the box walls: exercises every
    branch of fraction_inside."""
    phi = box_walls_phi(ni, nj, nk, h)
    lx, ly, lz = ni * h, nj * h, nk * h
    for _ in range(n_spheres):
        c = rng.uniform(0.2, 0.8, 3) * np.array([lx, ly, lz])
        r = rng.uniform(0.05, 0.25) * min(lx, ly, lz)
        phi = np.minimum(phi, sphere_phi(ni, nj, nk, h, c, r))
    return phi.astype(np.float32)


def face_shapes(ni, nj, nk):
    return (nk, nj, ni + 1), (nk, nj + 1, ni), (nk + 1, nj, ni)


def random_velocity(ni, nj, nk, rng, scale=1.0):
    su, sv, sw = face_shapes(ni, nj, nk)
    return tuple((scale * rng.standard_normal(s)).astype(np.float32) for s in (su, sv, sw))


def projection_problem(ni, nj, nk, seed=0, n_spheres=3, inflow=False, solid_velocity=False):
    """Inputs of one pressure projection (SmokeSolver3D::pcg_projection)."""
    rng = np.random.default_rng(seed)
    h = np.float32(1.0 / max(ni, nj, nk))
    phi = random_phi(ni, nj, nk, h, rng, n_spheres)
    u, v, w = random_velocity(ni, nj, nk, rng)
    su, sv, sw = face_shapes(ni, nj, nk)
    if solid_velocity:
        us, vs, ws = (0.1 * rng.standard_normal(s).astype(np.float32) for s in (su, sv, sw))
    else:
        us, vs, ws = (np.zeros(s, np.float32) for s in (su, sv, sw))
    bdesc = np.zeros((nk, nj, ni), np.int8)
    if inflow:
        bdesc[nk // 3:2 * nk // 3, nj // 3:2 * nj // 3, 1:3] = 1
    return dict(ni=ni, nj=nj, nk=nk, h=float(h), U_in=1.5, phi=phi, bdesc=bdesc, us=us, vs=vs, ws=ws,
                u=u, v=v, w=w)


def poisson_stencil(ni, nj, nk, h, uw, vw, ww):
    """The 7-slot operator pcg_projection assembles from face weights
    (Smoke_solver3D.cpp:986-1111) as float64 arrays (7, nk, nj, ni); for
    synthetic solver tests without the velocity part."""
    st = np.zeros((7, nk, nj, ni), np.float64)
    h2 = np.float32(h) * np.float32(h)
    k, j, i = np.meshgrid(np.arange(1, nk - 1), np.arange(1, nj - 1), np.arange(1, ni - 1), indexing="ij")
    t1 = (uw[k, j, i + 1] / h2).astype(np.float32)
    t2 = (uw[k, j, i] / h2).astype(np.float32)
    t3 = (vw[k, j + 1, i] / h2).astype(np.float32)
    t4 = (vw[k, j, i] / h2).astype(np.float32)
    t5 = (ww[k + 1, j, i] / h2).astype(np.float32)
    t6 = (ww[k, j, i] / h2).astype(np.float32)
    d = t1.astype(np.float64)
    for t in (t2, t3, t4, t5, t6):
        d = d + t.astype(np.float64)
    st[0, k, j, i] = d
    st[2, k, j, i] = np.where(i < ni - 2, -t1, 0)
    st[1, k, j, i] = np.where(i >= 2, -t2, 0)
    st[4, k, j, i] = np.where(j < nj - 2, -t3, 0)
    st[3, k, j, i] = np.where(j >= 2, -t4, 0)
    st[6, k, j, i] = np.where(k < nk - 2, -t5, 0)
    st[5, k, j, i] = np.where(k >= 2, -t6, 0)
    return st


def uniform_laplacian(ni, nj, nk):
    """Unit 7-point Laplacian on the interior with the Dirichlet ring of
    pcg_projection (ring rows empty, couplings to the ring dropped)."""
    o = np.ones((nk + 1, nj + 1, ni + 1), np.float32)
    uw, vw, ww = o[:nk, :nj, :ni + 1], o[:nk, :nj + 1, :ni], o[:nk + 1, :nj, :ni]
    return poisson_stencil(ni, nj, nk, 1.0, uw, vw, ww)


def random_particles(ni, nj, nk, h, n, rng, margin=1.0):
    """n particles uniformly in the domain (widened by `margin` cells on each
    side so out-of-range hashing is exercised), N(0,1) velocities."""
    p = np.zeros(n, PARTICLE_DTYPE)
    lo = -margin * h
    hi = np.array([ni, nj, nk]) * h + margin * h
    p["pos"] = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    p["vel"] = rng.standard_normal((n, 3)).astype(np.float32)
    return p


def jittered_particles(ni, nj, nk, h, ppc, rng, centre=None, radius=None):
    """ppc particles per cell, each uniformly jittered within its cell; with
    centre/radius only cells whose centre lies inside that sphere are seeded
    (the FLIP smoke source)."""
    k, j, i = np.meshgrid(np.arange(nk), np.arange(nj), np.arange(ni), indexing="ij")
    cells = np.stack([i.ravel(), j.ravel(), k.ravel()], 1).astype(np.float64)
    if centre is not None:
        d = np.linalg.norm(cells * h - np.asarray(centre), axis=1)
        cells = cells[d <= radius]
    n = len(cells) * ppc
    p = np.zeros(n, PARTICLE_DTYPE)
    base = np.repeat(cells, ppc, axis=0) * h
    p["pos"] = (base + rng.uniform(-0.49, 0.49, (n, 3)) * h).astype(np.float32)
    return p


def nested_scene(seed=0, dims=(20, 18, 16), h=1 / 32, lo=(5, 4, 4), cells=(10, 9, 8), ratio=2, scale=1.0):
    """A main grid with a nested subdomain (SmokeSolver3D + SubDomainSolver):
    main cells `dims` at spacing h with walls and a solid sphere; the
    subdomain covers main cells lo .. lo + cells at spacing h / ratio (its
    origin bmin = lo h), with its own random velocity and the same sphere in
    its own nodal phi.  Returns dict(dims, h, u, v, w, phi, sub) where sub is
    dict(dims, h, bmin, u, v, w, phi)."""
    rng = np.random.default_rng(seed)
    ni, nj, nk = dims
    h = np.float32(h)
    u, v, w = random_velocity(ni, nj, nk, rng, scale)
    bmin = (np.asarray(lo, np.float64) * h).astype(np.float32)
    sh = np.float32(h / ratio)
    sdims = tuple(int(c) * ratio for c in cells)
    # a sphere cutting the subdomain's box near one corner
    centre = bmin + np.float32(0.35) * np.asarray(cells, np.float32) * h
    radius = 0.22 * min(cells) * float(h)
    phi = np.minimum(box_walls_phi(ni, nj, nk, h), sphere_phi(ni, nj, nk, h, centre, radius)).astype(np.float32)
    su, sv, sw = random_velocity(*sdims, rng, scale)
    sphi = sphere_phi(*sdims, sh, centre - bmin, radius)
    sub = dict(dims=sdims, h=sh, bmin=bmin, u=su, v=sv, w=sw, phi=sphi)
    return dict(dims=(ni, nj, nk), h=h, u=u, v=v, w=w, phi=phi, sub=sub, rng=rng)


BATCH_SIDES = (32, 48, 64, 96, 128, 160, 192)


def batch_system(solver, side, seed, device=None):
    """One system of the batched uneven-Poisson workload: a side^3 box, 1-6
    random solid spheres of radius 0.05-0.25 side (nodal level set), and the
    rhs of the projection of an FP32 Gaussian velocity (sigma 1) smoothed by
    3 Jacobi sweeps (7-point averaging), assembled by the library's own
    projection assembly.  Returns (stencil[4, n, n, n], rhs[n, n, n]) on the
    device.  The random fields are generated on the GPU (torch, seeded)."""
    import torch

    rng = np.random.default_rng(seed)
    n = int(side)
    h = np.float32(1.0 / n)
    dev = solver.device if device is None else device
    phi = np.full((n + 1, n + 1, n + 1), 1.0, np.float32)
    for _ in range(int(rng.integers(1, 7))):
        c = rng.uniform(0.15, 0.85, 3)
        r = rng.uniform(0.05, 0.25)
        phi = np.minimum(phi, sphere_phi(n, n, n, h, c, r))
    g = torch.Generator(device=dev).manual_seed(int(seed))

    def smooth(a):
        for _ in range(3):
            p = torch.nn.functional.pad(a[None, None], (1, 1, 1, 1, 1, 1), mode="replicate")[0, 0]
            a = (p[1:-1, 1:-1, 1:-1] + p[:-2, 1:-1, 1:-1] + p[2:, 1:-1, 1:-1] + p[1:-1, :-2, 1:-1] +
                 p[1:-1, 2:, 1:-1] + p[1:-1, 1:-1, :-2] + p[1:-1, 1:-1, 2:]) / 7.0
        return a.contiguous()

    su, sv, sw = face_shapes(n, n, n)
    u, v, w = (smooth(torch.randn(s, generator=g, device=dev, dtype=torch.float32)) for s in (su, sv, sw))
    zeros = [torch.zeros(s, dtype=torch.float32, device=dev) for s in (su, sv, sw)]
    bdesc = torch.zeros((n, n, n), dtype=torch.int8, device=dev)
    st, rhs = solver.assemble(n, n, n, float(h), 0.0, torch.from_numpy(phi).to(dev), bdesc, *zeros, u, v, w)
    return st, rhs


def batch_workload(solver, count=32, seed=0, sides=BATCH_SIDES):
    """`count` systems with sides drawn uniformly from `sides` (seeded)."""
    rng = np.random.default_rng(seed)
    picks = rng.choice(np.asarray(sides), size=count)
    return [batch_system(solver, int(s), seed * 1000 + i) for i, s in enumerate(picks)], [int(s) for s in picks]
