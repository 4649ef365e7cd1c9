"""FLIP smoke stepper built from the library's kernels (the particle half of
the reference's SmokeSolver3D::time_step, SS/Smoke_solver3D.cpp:324-416).

One step, in the reference's order:
  1. advect_FLIP: RK3 through the grid velocity + solid push-out
     (vflip_advect_flip);
  2. hash_FLIP + particle_to_grid x3: sorted segmented P2G (vflip_p2g);
  3. the emitter: faces inside the source sphere get the inflow velocity
     (scene code; the reference emits through its particle sources);
  4. pcg_projection with plain MGPCG (vflip_project);
  5. compute_delta_u + particle_from_grid with the FLIP/PIC blend
     (vflip_delta, vflip_g2p);
  6. reorder_FLIP: 8 particles per open cell (vflip_reorder_flip).
The particle state (40-byte records) stays on the device.

With ``smoke=True`` the density/temperature block of time_step
(Smoke_solver3D.cpp:353-369) runs between steps 1 and 2: advect_field (RK3)
of density and temperature on their 2n^3 grid at h/2 along one shared
backtrace (vflip_advect_rk3_linear2), gen_heat (vflip_gen_heat) and the
buoyancy add_smokeforce on the particles (vflip_add_smokeforce).

With ``tracers_per_step > 0`` the tracer block of time_step runs first:
emit_tracers (the emitter at the source sphere) and advect_tracers through
the grid velocity (Smoke_solver3D.cpp:330-336, Smoke_solver3D.h:46-120);
``write_tracers`` stores them in the reference's Particle_data%04d.bin form.

``NestedFlipSim`` adds the nested subdomain (SubDomainSolver) and its
coupling, in time_step's order (Smoke_solver3D.cpp:324-411): the
subdomain's particles join the main set; advect_FLIP (and the tracers) use
the main grid's samplers with the subdomain active (vflip_*_nested: blended
get_velocity, the subdomain's solid phi and normal); after the main
projection and G2P the halo particles become the subdomain's, which runs its
own P2G, projection (dt 1, tolerance 1e-9, 1000 iterations), delta, G2P and
reorder (vflip_sub_*, vflip_project_subdomain); then the main reorder
filters on the nested solid phi.
"""
from dataclasses import dataclass

import numpy as np
import torch

from . import scenes
from .particles import PARTICLE_BYTES, PARTICLE_DTYPE


@dataclass
class FlipParams:
    n: int = 128
    dt: float = 0.01
    ppc: int = 8
    obstacle_centre: tuple = (0.5, 0.5, 0.5)
    obstacle_radius: float = 0.15
    source_centre: tuple = (0.5, 0.1, 0.5)
    source_radius: float = 0.12
    inflow: float = 1.0
    flip_ratio: float = 0.95
    tol: float = 1e-6
    max_iterations: int = 50
    seed: int = 0
    # density/temperature on the doubled grid (SmokeSolver3D::gen_heat and
    # add_smokeforce parameters, Smoke_solver3D.h:165-170)
    smoke: bool = False
    smoke_centre: tuple = (0.5, 0.1, 0.5)
    smoke_radius: float = 0.12
    smoke_dens: float = 1.0
    smoke_heat: float = 1.0
    dens_decay: float = 0.0
    temp_decay: float = 0.0
    alpha: float = 0.0
    beta: float = 1.0
    # tracers emitted per step in the source sphere (0: no tracers)
    tracers_per_step: int = 0

    @property
    def h(self):
        return float(np.float32(1.0 / self.n))


class FlipSim:
    def __init__(self, solver, params: FlipParams):
        self.s = solver
        self.p = params
        n, h, dev = params.n, np.float32(params.h), solver.device
        x, y, z = scenes.nodal_coords(n, n, n, h)
        self.phi = torch.from_numpy(self.solid_phi_at(x, y, z)).to(dev)
        su, sv, sw = scenes.face_shapes(n, n, n)
        self.shapes = (su, sv, sw)
        self.vel = [torch.zeros(s, dtype=torch.float32, device=dev) for s in (su, sv, sw)]
        self.solid = [torch.zeros(s, dtype=torch.float32, device=dev) for s in (su, sv, sw)]
        self.bdesc = torch.zeros((n, n, n), dtype=torch.int8, device=dev)
        self.pressure = torch.zeros((n, n, n), dtype=torch.float64, device=dev)
        rng = np.random.default_rng(params.seed)
        p = scenes.jittered_particles(n, n, n, h, params.ppc, rng, centre=params.source_centre,
                                      radius=params.source_radius)
        p["vel"][:, 1] = params.inflow
        self.particles = torch.from_numpy(p.view(np.uint8).copy()).to(dev)
        # v faces (world (ih, (j - 1/2)h, kh)) inside the source sphere
        k, j, i = np.meshgrid(np.arange(sv[0]), np.arange(sv[1]), np.arange(sv[2]), indexing="ij")
        c = params.source_centre
        d2 = (i * h - c[0]) ** 2 + ((j - 0.5) * h - c[1]) ** 2 + (k * h - c[2]) ** 2
        self.source_v = torch.from_numpy(d2 <= params.source_radius ** 2).to(dev)
        if params.smoke:
            self.rho = torch.zeros((2 * n,) * 3, dtype=torch.float32, device=dev)
            self.temp = torch.zeros_like(self.rho)
            self._rho2 = torch.empty_like(self.rho)
            self._temp2 = torch.empty_like(self.rho)
        self.tracers = torch.zeros((0, 4), dtype=torch.float32, device=dev)
        self.steps = 0
        self.last = None

    def solid_phi_at(self, x, y, z):
        """The scene's solid signed distance at world points: walls one cell
        thick on five faces (open top) and the obstacle sphere (none when its
        radius is 0); positive in the fluid."""
        p = self.p
        h = float(np.float32(p.h))
        L = p.n * h
        phi = np.minimum.reduce([x - h, (L - 2 * h) - x, y - h, z - h, (L - 2 * h) - z])
        if p.obstacle_radius > 0:
            c = p.obstacle_centre
            d = np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) - p.obstacle_radius
            phi = np.minimum(phi, d)
        return phi.astype(np.float32)

    @property
    def num_particles(self):
        return self.particles.numel() // PARTICLE_BYTES

    def particles_host(self):
        return self.particles.cpu().numpy().view(PARTICLE_DTYPE)

    def step(self):
        p, s, n, h = self.p, self.s, self.p.n, self.p.h
        u, v, w = self.vel
        if p.tracers_per_step > 0:
            L = float(np.float32(h) * n)
            self.tracers = s.emit_tracers(self.tracers if self.tracers.shape[0] else None, h, (L, L, L),
                                          p.source_centre, p.source_radius, p.tracers_per_step, seed=p.seed + self.steps)
            s.advect_tracers(n, n, n, h, self.tracers, u, v, w, self.phi, p.dt, p.dens_decay)
        s.advect_flip(n, n, n, h, self.particles, u, v, w, self.phi, p.dt)
        if p.smoke:
            self.smoke_scalars(u, v, w)
        outs = s.particle_to_grid(n, n, n, h, self.particles)
        un, vn, wn = outs[0][0], outs[1][0], outs[2][0]
        vn.masked_fill_(self.source_v, p.inflow)
        before = [un.clone(), vn.clone(), wn.clone()]
        conv, _, stats = s.project(n, n, n, h, 0.0, self.phi, self.bdesc, *self.solid, un, vn, wn,
                                   pressure=self.pressure, tolerance_factor=p.tol, max_iterations=p.max_iterations)
        delta = [s.delta(a, b) for a, b in zip((un, vn, wn), before)]
        s.particle_from_grid(n, n, n, h, self.particles, *delta, un, vn, wn, flip_ratio=p.flip_ratio)
        self.particles = s.reorder_flip(n, n, n, h, self.particles, un, vn, wn, self.phi, seed=p.seed + self.steps)
        self.vel = [un, vn, wn]
        self.steps += 1
        self.last = stats
        return conv, stats

    def smoke_scalars(self, u, v, w):
        """advect_field of density and temperature, gen_heat, add_smokeforce
        (Smoke_solver3D.cpp:358-369) through the grid velocity u, v, w."""
        p, s, n = self.p, self.s, self.p.n
        fh = self.p.h / 2
        s.advect_rk3_linear(n, n, n, p.h, p.dt, u, v, w, self.rho, fh, field2=self.temp, out=self._rho2,
                            out2=self._temp2)
        self.rho, self._rho2 = self._rho2, self.rho
        self.temp, self._temp2 = self._temp2, self.temp
        s.gen_heat(self.rho, self.temp, fh, p.dt, p.dens_decay, p.temp_decay, p.smoke_centre, p.smoke_radius,
                   p.smoke_dens, p.smoke_heat)
        s.add_smokeforce(self.particles, self.rho, self.temp, fh, p.alpha, p.beta, p.dt)

    def write_tracers(self, directory, frame):
        """The tracers as <directory>/Particle_data%04d.bin (SmokeSolver3D::write_tracers)."""
        self.s.write_tracers(self.tracers, float(np.float32(self.p.h) * self.p.n), directory, frame)


@dataclass
class NestedParams(FlipParams):
    # the subdomain covers main cells sub_lo .. sub_lo + sub_cells at spacing
    # h / ratio (defaults: the central half at 2x refinement)
    sub_lo: tuple = None
    sub_cells: tuple = None
    ratio: int = 2
    sub_tol: float = 1e-9
    sub_max_iterations: int = 1000


class NestedFlipSim(FlipSim):
    def __init__(self, solver, params: NestedParams):
        if params.smoke:
            raise ValueError("the density/temperature block is not coupled to the subdomain")
        super().__init__(solver, params)
        p, dev, n = params, solver.device, params.n
        h = np.float32(p.h)
        lo = p.sub_lo if p.sub_lo is not None else (n // 4,) * 3
        cells = p.sub_cells if p.sub_cells is not None else (n // 2,) * 3
        self.sh = np.float32(h / p.ratio)
        self.sdims = tuple(int(c) * p.ratio for c in cells)
        self.bmin = tuple(float(np.float32(np.float32(l) * h)) for l in lo)
        sni, snj, snk = self.sdims
        x, y, z = scenes.nodal_coords(sni, snj, snk, self.sh)
        self.sphi = torch.from_numpy(self.solid_phi_at(x + np.float32(self.bmin[0]), y + np.float32(self.bmin[1]),
                                                       z + np.float32(self.bmin[2]))).to(dev)
        shapes = scenes.face_shapes(sni, snj, snk)
        self.sub_vel = [torch.zeros(sh, dtype=torch.float32, device=dev) for sh in shapes]
        self.sub_solid = [torch.zeros(sh, dtype=torch.float32, device=dev) for sh in shapes]
        self.sub_pressure = torch.zeros((snk, snj, sni), dtype=torch.float64, device=dev)
        self.sub_desc = solver.subdomain(self.sdims, self.sh, self.bmin, *self.sub_vel, self.sphi)
        # SubDomainSolver::init (sub_domain.h:161-175) ends with hash_FLIP +
        # reorder_FLIP of an empty set: 8 particles per interior cell, at rest
        empty = torch.zeros(0, dtype=torch.uint8, device=dev)
        self.sub_particles = solver.sub_reorder_flip(sni, snj, snk, self.sh, self.bmin, empty, *self.sub_vel,
                                                     self.sphi, seed=p.seed ^ 0x5EED)
        self.last_sub = None

    @property
    def num_sub_particles(self):
        return self.sub_particles.numel() // PARTICLE_BYTES

    def step(self):
        p, s, n, h = self.p, self.s, self.p.n, self.p.h
        sni, snj, snk = self.sdims
        u, v, w = self.vel
        seed = p.seed + self.steps
        if p.tracers_per_step > 0:
            L = float(np.float32(h) * n)
            self.tracers = s.emit_tracers_nested(self.tracers if self.tracers.shape[0] else None, h, (L, L, L),
                                                 p.source_centre, p.source_radius, p.tracers_per_step, (n, n, n),
                                                 self.phi, self.sub_desc, seed=seed)
            s.advect_tracers_nested(n, n, n, h, self.tracers, u, v, w, self.phi, p.dt, p.dens_decay, self.sub_desc)
        # FLIP += sub_domain.FLIP, then the main particle pass
        if self.sub_particles.numel():
            self.particles = torch.cat([self.particles, self.sub_particles])
        s.advect_flip_nested(n, n, n, h, self.particles, u, v, w, self.phi, p.dt, self.sub_desc)
        outs = s.particle_to_grid(n, n, n, h, self.particles)
        un, vn, wn = outs[0][0], outs[1][0], outs[2][0]
        vn.masked_fill_(self.source_v, p.inflow)
        before = [un.clone(), vn.clone(), wn.clone()]
        conv, _, stats = s.project(n, n, n, h, 0.0, self.phi, self.bdesc, *self.solid, un, vn, wn,
                                   pressure=self.pressure, tolerance_factor=p.tol, max_iterations=p.max_iterations)
        delta = [s.delta(a, b) for a, b in zip((un, vn, wn), before)]
        s.particle_from_grid(n, n, n, h, self.particles, *delta, un, vn, wn, flip_ratio=p.flip_ratio)
        # the subdomain's pass on the halo particles
        self.sub_particles = s.halo_select(self.particles, h, self.sub_desc)
        so = s.sub_particle_to_grid(sni, snj, snk, self.sh, self.bmin, self.sub_particles)
        su, sv, sw = so[0][0], so[1][0], so[2][0]
        sbefore = [su.clone(), sv.clone(), sw.clone()]
        sconv, _, sstats = s.project_subdomain(sni, snj, snk, self.sh, 1.0, self.sphi, *self.sub_solid, su, sv, sw,
                                               pressure=self.sub_pressure, tolerance_factor=p.sub_tol,
                                               max_iterations=p.sub_max_iterations)
        sdelta = [s.delta(a, b) for a, b in zip((su, sv, sw), sbefore)]
        s.sub_particle_from_grid(sni, snj, snk, self.sh, self.bmin, self.sub_particles, *sdelta)
        self.sub_particles = s.sub_reorder_flip(sni, snj, snk, self.sh, self.bmin, self.sub_particles, su, sv, sw,
                                                self.sphi, seed=seed ^ 0x5EED)
        self.sub_vel = [su, sv, sw]
        self.sub_desc = s.subdomain(self.sdims, self.sh, self.bmin, su, sv, sw, self.sphi)
        # the main reorder, filtered on the nested solid phi
        self.particles = s.reorder_flip_nested(n, n, n, h, self.particles, un, vn, wn, self.phi, self.sub_desc,
                                               seed=seed)
        self.vel = [un, vn, wn]
        self.steps += 1
        self.last, self.last_sub = stats, sstats
        return conv and sconv, stats, sstats
