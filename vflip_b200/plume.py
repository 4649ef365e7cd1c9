"""Grid smoke-plume stepper built from the library's kernels.

One step (the unit of the benchmark) is one smoke step:
  1. RK2 semi-Lagrangian trilinear advection of u, v, w (one launch) and of
     density and temperature (one launch, one shared backtrace) through the
     current velocity (SubDomainSolver::advect_field, sub_domain.cpp:191-235);
  2. density/temperature source sphere and buoyancy on the v faces (grid
     analogue of gen_heat / add_smokeforce, Smoke_solver3D.cpp:1624-1668);
  3. pressure projection with MGPCG to the tolerance
     (SmokeSolver3D::pcg_projection, Smoke_solver3D.cpp:945-1202).

Solids are the five box walls (open top) and optionally the centred sphere
obstacle, as a nodal level set.
"""
from dataclasses import dataclass

import numpy as np
import torch

from . import scenes


@dataclass
class PlumeParams:
    n: int
    dt: float = 0.01
    obstacle: bool = True
    obstacle_centre: tuple = (0.5, 0.5, 0.5)
    obstacle_radius: float = 0.15
    source_centre: tuple = (0.5, 0.1, 0.5)
    source_radius: float = 0.1
    alpha: float = 0.1
    beta: float = 1.0
    tol: float = 1e-6
    max_iterations: int = 50

    @property
    def h(self):
        return float(np.float32(1.0 / self.n))


def nodal_phi(p: PlumeParams):
    n, h = p.n, np.float32(p.h)
    phi = scenes.box_walls_phi(n, n, n, h, open_top=True)
    if p.obstacle:
        phi = np.minimum(phi, scenes.sphere_phi(n, n, n, h, p.obstacle_centre, p.obstacle_radius))
    return phi.astype(np.float32)


class PlumeSim:
    FIELDS = ("u", "v", "w", "rho", "temp")

    def __init__(self, solver, params: PlumeParams):
        self.s = solver
        self.p = params
        n = params.n
        dev = solver.device
        su, sv, sw = scenes.face_shapes(n, n, n)
        shapes = {"u": su, "v": sv, "w": sw, "rho": (n, n, n), "temp": (n, n, n)}
        self.shapes = shapes
        self.f = {k: torch.zeros(shapes[k], dtype=torch.float32, device=dev) for k in self.FIELDS}
        self.g = {k: torch.zeros(shapes[k], dtype=torch.float32, device=dev) for k in self.FIELDS}
        self.phi = torch.from_numpy(nodal_phi(params)).to(dev)
        self.bdesc = torch.zeros((n, n, n), dtype=torch.int8, device=dev)
        self.solid = {k: torch.zeros(shapes[k], dtype=torch.float32, device=dev) for k in ("u", "v", "w")}
        self.pressure = torch.zeros((n, n, n), dtype=torch.float64, device=dev)
        self.last = None

    def load_state(self, arrays):
        for k in self.FIELDS:
            self.f[k].copy_(torch.as_tensor(arrays[k]), non_blocking=True)

    def state(self):
        return {k: self.f[k] for k in self.FIELDS}

    def advect_and_force(self, before_scalars=None):
        """Steps 1-2 of a plume step (advection, sources, buoyancy);
        `before_scalars` runs between the velocity and the scalar advection."""
        p, s, n, h = self.p, self.s, self.p.n, self.p.h
        u, v, w = self.f["u"], self.f["v"], self.f["w"]
        s.advect_velocity_rk2_linear(n, n, n, h, p.dt, u, v, w, outs=(self.g["u"], self.g["v"], self.g["w"]))
        if before_scalars is not None:
            before_scalars()
        # density and temperature share the cell-centred backtrace
        s.advect_rk2_linear2(n, n, n, h, p.dt, u, v, w, self.f["rho"], self.f["temp"], (0, 0, 0), out=self.g["rho"],
                             out2=self.g["temp"])
        self.f, self.g = self.g, self.f
        s.plume_sources(n, n, n, h, p.dt, self.f["rho"], self.f["temp"], self.f["v"], p.source_centre,
                        p.source_radius, 1.0, 1.0, p.alpha, p.beta)

    def project(self, solver=None, u=None, v=None, w=None, pressure=None):
        """Step 3: the pressure projection of (u, v, w) (the state by default)."""
        p, n, h = self.p, self.p.n, self.p.h
        s = solver or self.s
        u = self.f["u"] if u is None else u
        v = self.f["v"] if v is None else v
        w = self.f["w"] if w is None else w
        pressure = self.pressure if pressure is None else pressure
        return s.project(n, n, n, h, 0.0, self.phi, self.bdesc, self.solid["u"], self.solid["v"], self.solid["w"], u,
                         v, w, pressure=pressure, tolerance_factor=p.tol, max_iterations=p.max_iterations)

    def project_learned(self, net, mode, level, sample=None):
        """Step 3 through vflip_project_learned (capture or learned solve)."""
        p, n, h = self.p, self.p.n, self.p.h
        return self.s.project_learned(net, mode, level, n, n, n, h, 0.0, self.phi, self.bdesc, self.solid["u"],
                                      self.solid["v"], self.solid["w"], self.f["u"], self.f["v"], self.f["w"],
                                      pressure=self.pressure, tolerance_factor=p.tol,
                                      max_iterations=p.max_iterations, sample=sample)

    def step(self, precond=None, before_scalars=None, after_force=None):
        """One plume step; `precond` (a learned.LearnedPreconditioner) takes
        over the projection when given.  `before_scalars` / `after_force` run
        before the scalar advection / before the projection."""
        self.advect_and_force(before_scalars)
        if after_force is not None:
            after_force()
        if precond is None:
            conv, _, stats = self.project()
        else:
            conv, stats = precond.project(self)
        self.last = stats
        return conv, stats

    def divergence(self, u, v, w):
        """Weighted discrete divergence sum(w_f u_f n_f)/h per cell, the
        quantity the projection drives to zero, on the cells two or more
        away from the Dirichlet ring (the reference leaves the faces next to
        the ring uncorrected, Smoke_solver3D.cpp:1135)."""
        uw, vw, ww = self.s.face_weights(self.p.n, self.p.n, self.p.n, self.phi)
        h = self.p.h
        fu, fv, fw = uw * u, vw * v, ww * w
        div = (fu[:, :, 1:] - fu[:, :, :-1] + fv[:, 1:, :] - fv[:, :-1, :] + fw[1:, :, :] - fw[:-1, :, :]) / h
        return div[2:-2, 2:-2, 2:-2]

    def step_host(self, host, precond=None):
        """One step on host-resident state (pinned tensors): every field is
        copied in at the start of the step and its result copied back into
        the same host tensors.  The copies overlap the compute where the data
        allows:
          * u, v, w download in order on one stream, in HOST_CHUNKS pieces
            each, and each piece's next upload waits only for its own
            download, so uploads run one piece behind the downloads (the host
            link is full duplex);
          * density and temperature travel on a third stream: their upload
            follows the velocity's and overlaps the velocity advection, their
            download leaves once the sources are applied and overlaps the
            projection.
        The step returns with its velocity downloads in flight: call
        host_join() before reading the host state or stopping a clock."""
        dev = self.s.device
        main = torch.cuda.current_stream(dev)
        if getattr(self, "_up", None) is None:
            self._up, self._down, self._cs = (torch.cuda.Stream(dev) for _ in range(3))
            self._downloaded = {}
        up, down, cs = self._up, self._down, self._cs
        up.wait_stream(main)  # the device buffers are free of earlier work
        with torch.cuda.stream(up):
            for k in ("u", "v", "w"):
                for c, (d, h) in enumerate(zip(self._pieces(self.f[k]), self._pieces(host[k]))):
                    if (k, c) in self._downloaded:
                        up.wait_event(self._downloaded[(k, c)])
                    d.copy_(h, non_blocking=True)
        vel_in = torch.cuda.Event()
        vel_in.record(up)
        main.wait_event(vel_in)
        cs.wait_event(vel_in)
        with torch.cuda.stream(cs):
            for k in ("rho", "temp"):
                self.f[k].copy_(host[k], non_blocking=True)
        scal_in = torch.cuda.Event()
        scal_in.record(cs)

        def download_scalars():
            cs.wait_stream(main)
            with torch.cuda.stream(cs):
                for k in ("rho", "temp"):
                    host[k].copy_(self.f[k], non_blocking=True)

        out = self.step(precond, before_scalars=lambda: main.wait_event(scal_in), after_force=download_scalars)
        down.wait_stream(main)
        with torch.cuda.stream(down):
            for k in ("u", "v", "w"):
                for c, (d, h) in enumerate(zip(self._pieces(self.f[k]), self._pieces(host[k]))):
                    h.copy_(d, non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(down)
                    self._downloaded[(k, c)] = ev
        return out

    HOST_CHUNKS = 8

    def _pieces(self, t):
        """HOST_CHUNKS contiguous pieces of a field (flat views)."""
        flat = t.view(-1)
        n = flat.numel()
        bounds = [n * c // self.HOST_CHUNKS for c in range(self.HOST_CHUNKS + 1)]
        return [flat[a:b] for a, b in zip(bounds[:-1], bounds[1:])]

    def host_join(self):
        """Make the current stream wait for step_host's copies in flight."""
        main = torch.cuda.current_stream(self.s.device)
        for st in (getattr(self, "_down", None), getattr(self, "_cs", None), getattr(self, "_up", None)):
            if st is not None:
                main.wait_stream(st)

    def host_bytes(self):
        return sum(int(np.prod(self.shapes[k])) * 4 for k in self.FIELDS)
