"""Host-side mirror of the reference's solver call surface over the C ABI.

``Solver`` owns one ``vflip_ctx`` (device buffers, PCG scalars, a stream:
torch's current stream by default, so the library's kernels are ordered with
the caller's torch work).  Methods take torch CUDA tensors and return
torch CUDA tensors; ``amgpcg_solve_csr`` is the exact drop-in of
``ivock::AMGPCGSolve`` and takes host (numpy) arrays like the reference.

Status handling mirrors the reference: the solve returns the reference's bool
(converged or not) plus residual and iteration count; argument and CUDA
errors raise ``VflipError``.
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from ._lib import ConfigC, LearnedStatsC, SolveStatsC, SubdomainC, SystemC, VflipError, load
from .particles import PARTICLE_BYTES


@dataclass
class SolveStats:
    iterations: int
    vcycles: int
    levels: int
    converged: bool
    residual: float
    rhs_norm: float
    solve_ms: float

    @classmethod
    def from_c(cls, s):
        return cls(s.iterations, s.vcycles, s.levels, bool(s.converged), s.residual, s.rhs_norm, s.solve_ms)


@dataclass
class LearnedStats:
    fallback: bool
    subspace: int
    gamma: tuple
    init_residual: float
    net_ms: float

    @classmethod
    def from_c(cls, s):
        return cls(bool(s.fallback), s.subspace, tuple(s.gamma), s.init_residual, s.net_ms)


def _p(t):
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return C.c_void_p(t.ctypes.data)
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return C.c_void_p(t.data_ptr())


def _face_shapes(ni, nj, nk):
    return (nk, nj, ni + 1), (nk, nj + 1, ni), (nk + 1, nj, ni)


class Solver:
    def __init__(self, precision=1, pre_sweeps=4, post_sweeps=4, coarse_sweeps=0, coarsest_max_unknowns=0,
                 device=0, stream=None, sweep_kernel=0, smoother_depth=0, smoother_tile_rows=0,
                 smoother_plane_ranges=0, smoother_ctas_per_sm=0, smoother_threads=0,
                 smoother_prefetch=0, coarsest_solver=0, spmv_kernel=0, pcg_loop=0, pcg_vectors=0,
                 batch_chunk=0, batch_ctas_per_sm=0, coarse_tail=0, tile_sweep_max_cells=0,
                 p2g_kernel=0, advect_kernel=0):
        self.lib = load()
        cfg = ConfigC()
        self.lib.vflip_config_default(C.byref(cfg))
        cfg.precision = precision
        cfg.pre_sweeps = pre_sweeps
        cfg.post_sweeps = post_sweeps
        cfg.coarse_sweeps = coarse_sweeps
        cfg.coarsest_max_unknowns = coarsest_max_unknowns
        cfg.device = device
        cfg.sweep_kernel = sweep_kernel
        cfg.smoother_depth = smoother_depth
        cfg.smoother_tile_rows = smoother_tile_rows
        cfg.smoother_plane_ranges = smoother_plane_ranges
        cfg.smoother_ctas_per_sm = smoother_ctas_per_sm
        cfg.smoother_threads = smoother_threads
        cfg.smoother_prefetch = smoother_prefetch
        cfg.coarsest_solver = coarsest_solver
        cfg.spmv_kernel = spmv_kernel
        cfg.pcg_loop = pcg_loop
        cfg.pcg_vectors = pcg_vectors
        cfg.batch_chunk = batch_chunk
        cfg.batch_ctas_per_sm = batch_ctas_per_sm
        cfg.coarse_tail = coarse_tail
        cfg.tile_sweep_max_cells = tile_sweep_max_cells
        cfg.p2g_kernel = p2g_kernel
        cfg.advect_kernel = advect_kernel
        self.device = torch.device("cuda", device)
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        self.stream = stream
        cfg.stream = C.c_void_p(stream.cuda_stream)
        ctx = C.c_void_p()
        rc = self.lib.vflip_create(C.byref(ctx), C.byref(cfg))
        if rc != 0:
            raise VflipError(rc, "vflip_create failed")
        self.ctx = ctx
        self.precision = precision

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.vflip_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------- helpers
    def _check(self, rc):
        if rc < 0:
            raise VflipError(rc, self.lib.vflip_last_error(self.ctx).decode())
        return rc

    def _empty(self, shape, dtype):
        return torch.empty(shape, dtype=dtype, device=self.device)

    def synchronize(self):
        self._check(self.lib.vflip_synchronize(self.ctx))

    @property
    def last_ms(self):
        return self.lib.vflip_last_ms(self.ctx)

    # ------------------------------------------------------------- MGPCG
    def amgpcg_solve_csr(self, rowstart, colindex, value, rhs, tolerance_factor, max_iterations, ni, nj, nk):
        """Drop-in of ivock::AMGPCGSolve on host CSR arrays.  Returns
        (success, result, residual_out, iterations_out)."""
        rowstart = np.ascontiguousarray(rowstart, np.uint32)
        colindex = np.ascontiguousarray(colindex, np.uint32)
        value = np.ascontiguousarray(value, np.float64)
        rhs = np.ascontiguousarray(rhs, np.float64).ravel()
        result = np.zeros_like(rhs)
        res = C.c_double(0.0)
        it = C.c_int(0)
        rc = self.lib.vflip_amgpcg_solve_csr(self.ctx, len(rhs), _p(rowstart), _p(colindex), _p(value), _p(rhs),
                                            _p(result), float(tolerance_factor), int(max_iterations), C.byref(res),
                                            C.byref(it), ni, nj, nk)
        self._check(rc)
        return rc == 0, result, res.value, it.value

    def amgpcg_solve(self, stencil, rhs, tolerance_factor=1e-6, max_iterations=50, result=None):
        """Solve A p = rhs for a (4, nk, nj, ni) float64 stencil (diag, xp,
        yp, zp) on the device.  Returns (converged, result, SolveStats)."""
        _, nk, nj, ni = stencil.shape
        if result is None:
            result = self._empty((nk, nj, ni), torch.float64)
        st = SolveStatsC()
        rc = self.lib.vflip_amgpcg_solve(self.ctx, ni, nj, nk, _p(stencil[0]), _p(stencil[1]), _p(stencil[2]),
                                        _p(stencil[3]), _p(rhs), _p(result), float(tolerance_factor),
                                        int(max_iterations), C.byref(st))
        self._check(rc)
        return rc == 0, result, SolveStats.from_c(st)

    def build_levels(self, stencil, max_levels=16):
        _, nk, nj, ni = stencil.shape
        dims = np.zeros(3 * max_levels, np.int32)
        total, a, b, c = 0, ni, nj, nk
        for _ in range(max_levels):
            total += 4 * a * b * c
            a, b, c = (a + 1) // 2, (b + 1) // 2, (c + 1) // 2
        out = self._empty((total,), torch.float64)
        nl = self._check(self.lib.vflip_build_levels(self.ctx, ni, nj, nk, _p(stencil[0]), _p(stencil[1]),
                                                     _p(stencil[2]), _p(stencil[3]), max_levels, _p(dims),
                                                     _p(out)))
        levels, off = [], 0
        for l in range(nl):
            x, y, z = (int(v) for v in dims[3 * l:3 * l + 3])
            m = 4 * x * y * z
            levels.append(out[off:off + m].view(4, z, y, x))
            off += m
        return levels

    def rbgs(self, stencil, b, x, iterations):
        """In-place red-black Gauss-Seidel on float64 x."""
        _, nk, nj, ni = stencil.shape
        self._check(self.lib.vflip_rbgs(self.ctx, ni, nj, nk, _p(stencil[0]), _p(stencil[1]), _p(stencil[2]),
                                        _p(stencil[3]), _p(b), _p(x), int(iterations)))
        return x

    def vcycle(self, stencil, b):
        _, nk, nj, ni = stencil.shape
        x = self._empty((nk, nj, ni), torch.float64)
        self._check(self.lib.vflip_vcycle(self.ctx, ni, nj, nk, _p(stencil[0]), _p(stencil[1]), _p(stencil[2]),
                                          _p(stencil[3]), _p(b), _p(x)))
        return x

    # ------------------------------------------------------------- projection
    def face_weights(self, ni, nj, nk, nodal_phi):
        su, sv, sw = _face_shapes(ni, nj, nk)
        uw, vw, ww = self._empty(su, torch.float32), self._empty(sv, torch.float32), self._empty(sw, torch.float32)
        self._check(self.lib.vflip_face_weights(self.ctx, ni, nj, nk, _p(nodal_phi), _p(uw), _p(vw), _p(ww)))
        return uw, vw, ww

    def assemble(self, ni, nj, nk, h, U_in, nodal_phi, bdesc, us, vs, ws, u, v, w):
        st = self._empty((4, nk, nj, ni), torch.float64)
        rhs = self._empty((nk, nj, ni), torch.float64)
        self._check(self.lib.vflip_assemble(self.ctx, ni, nj, nk, float(h), float(U_in), _p(nodal_phi), _p(bdesc),
                                            _p(us), _p(vs), _p(ws), _p(u), _p(v), _p(w), _p(st[0]), _p(st[1]),
                                            _p(st[2]), _p(st[3]), _p(rhs)))
        return st, rhs

    def project(self, ni, nj, nk, h, U_in, nodal_phi, bdesc, us, vs, ws, u, v, w, pressure=None,
                tolerance_factor=1e-6, max_iterations=50):
        """SmokeSolver3D::pcg_projection on device arrays; u/v/w updated in
        place.  Returns (converged, pressure, SolveStats)."""
        if pressure is None:
            pressure = self._empty((nk, nj, ni), torch.float64)
        st = SolveStatsC()
        rc = self.lib.vflip_project(self.ctx, ni, nj, nk, float(h), float(U_in), _p(nodal_phi), _p(bdesc), _p(us),
                                   _p(vs), _p(ws), _p(u), _p(v), _p(w), _p(pressure), float(tolerance_factor),
                                   int(max_iterations), C.byref(st))
        self._check(rc)
        return rc == 0, pressure, SolveStats.from_c(st)

    def batched_solve(self, systems, tolerance_factor=1e-6, max_iterations=50, mode=0):
        """vflip_batched_solve over [(stencil[4, nk, nj, ni] float64, rhs[nk, nj, ni] float64), ...]
        (device tensors).  mode 0: one CUDA graph with device-side loops;
        1: one system after another; 2: one persistent cooperative kernel.  Returns (all_converged, [pressure], [SolveStats])."""
        n = len(systems)
        arr = (SystemC * max(n, 1))()
        results = []
        for i, (st, rhs) in enumerate(systems):
            nk, nj, ni = rhs.shape
            res = self._empty((nk, nj, ni), torch.float64)
            results.append(res)
            arr[i] = SystemC(ni, nj, nk, _p(st[0]).value, _p(st[1]).value, _p(st[2]).value, _p(st[3]).value,
                             _p(rhs).value, _p(res).value)
        stats = (SolveStatsC * max(n, 1))()
        rc = self.lib.vflip_batched_solve(self.ctx, n, arr, float(tolerance_factor), int(max_iterations), int(mode),
                                          stats)
        self._check(rc)
        return rc == 0, results, [SolveStats.from_c(stats[i]) for i in range(n)]

    def learned_grid(self, ni, nj, nk, level):
        X, Y, Z = C.c_int(), C.c_int(), C.c_int()
        self._check(self.lib.vflip_learned_grid(ni, nj, nk, level, C.byref(X), C.byref(Y), C.byref(Z)))
        return X.value, Y.value, Z.value

    def project_learned(self, net, mode, level, ni, nj, nk, h, U_in, nodal_phi, bdesc, us, vs, ws, u, v, w,
                        pressure=None, tolerance_factor=1e-6, max_iterations=50, sample=None):
        """vflip_project_learned.  mode: VFLIP_LEARNED_CAPTURE (1) with
        sample = (in2, target2, weight) tensors on the network grid, or
        VFLIP_LEARNED_SOLVE (2, | 4 to leave V(b) out of the Ritz step) with
        a ``learned.UNet``.  Returns (converged, pressure, SolveStats,
        LearnedStats)."""
        if pressure is None:
            pressure = self._empty((nk, nj, ni), torch.float64)
        st, ls = SolveStatsC(), LearnedStatsC()
        si, stt, sw = sample if sample is not None else (None, None, None)
        rc = self.lib.vflip_project_learned(self.ctx, net.h if net is not None else None, int(mode), int(level), ni, nj,
                                            nk, float(h), float(U_in), _p(nodal_phi), _p(bdesc), _p(us), _p(vs),
                                            _p(ws), _p(u), _p(v), _p(w), _p(pressure), float(tolerance_factor),
                                            int(max_iterations), _p(si), _p(stt), _p(sw), C.byref(st), C.byref(ls))
        self._check(rc)
        return rc == 0, pressure, SolveStats.from_c(st), LearnedStats.from_c(ls)

    def project_subdomain(self, ni, nj, nk, h, dt, nodal_phi, us, vs, ws, u, v, w, pressure=None,
                          tolerance_factor=1e-9, max_iterations=1000):
        """SubDomainSolver::pcg_projection (dt-scaled operator, tolerance 1e-9
        and 1000 iterations by default, as the reference calls it)."""
        if pressure is None:
            pressure = self._empty((nk, nj, ni), torch.float64)
        st = SolveStatsC()
        rc = self.lib.vflip_project_subdomain(self.ctx, ni, nj, nk, float(h), float(dt), _p(nodal_phi), _p(us),
                                              _p(vs), _p(ws), _p(u), _p(v), _p(w), _p(pressure),
                                              float(tolerance_factor), int(max_iterations), C.byref(st))
        self._check(rc)
        return rc == 0, pressure, SolveStats.from_c(st)

    # ------------------------------------------------------------- advection
    def advect_rk2_linear(self, ni, nj, nk, h, dt, u, v, w, field, offsets, out=None):
        fnz, fny, fnx = field.shape
        if out is None:
            out = torch.empty_like(field)
        self._check(self.lib.vflip_advect_rk2_linear(self.ctx, ni, nj, nk, float(h), float(dt), _p(u), _p(v), _p(w),
                                                     fnx, fny, fnz, float(offsets[0]), float(offsets[1]),
                                                     float(offsets[2]), _p(field), _p(out)))
        return out

    def advect_rk2_linear2(self, ni, nj, nk, h, dt, u, v, w, field, field2, offsets, out=None, out2=None):
        """Two fields on the same grid advected along one backtrace."""
        fnz, fny, fnx = field.shape
        out = torch.empty_like(field) if out is None else out
        out2 = torch.empty_like(field2) if out2 is None else out2
        self._check(self.lib.vflip_advect_rk2_linear2(self.ctx, ni, nj, nk, float(h), float(dt), _p(u), _p(v), _p(w),
                                                      fnx, fny, fnz, float(offsets[0]), float(offsets[1]),
                                                      float(offsets[2]), _p(field), _p(out), _p(field2), _p(out2)))
        return out, out2

    def advect_velocity_rk2_linear(self, ni, nj, nk, h, dt, u, v, w, outs=None):
        """SubDomainSolver::advect_field of u, v and w through themselves, one call."""
        outs = tuple(torch.empty_like(a) for a in (u, v, w)) if outs is None else outs
        self._check(self.lib.vflip_advect_velocity_rk2_linear(self.ctx, ni, nj, nk, float(h), float(dt), _p(u), _p(v),
                                                              _p(w), *[_p(o) for o in outs]))
        return outs

    def advect_cubic_clamp(self, ni, nj, nk, h, dt, u, v, w, field, offsets, out=None):
        """SmokeSolver3D::advect_field_cubic_clamp of one field."""
        fnz, fny, fnx = field.shape
        if out is None:
            out = torch.empty_like(field)
        self._check(self.lib.vflip_advect_cubic_clamp(self.ctx, ni, nj, nk, float(h), float(dt), _p(u), _p(v), _p(w),
                                                      fnx, fny, fnz, float(offsets[0]), float(offsets[1]),
                                                      float(offsets[2]), _p(field), _p(out)))
        return out

    def advect_velocity_cubic_clamp(self, ni, nj, nk, h, dt, u, v, w, outs=None):
        """SmokeSolver3D::advect: (u, v, w) advected by themselves, one launch."""
        outs = tuple(torch.empty_like(a) for a in (u, v, w)) if outs is None else outs
        self._check(self.lib.vflip_advect_velocity_cubic_clamp(self.ctx, ni, nj, nk, float(h), float(dt), _p(u),
                                                               _p(v), _p(w), *[_p(o) for o in outs]))
        return outs

    def advect_rk3_linear(self, ni, nj, nk, h, dt, u, v, w, field, fh, offsets=(0.0, 0.0, 0.0), field2=None,
                          out=None, out2=None):
        """SmokeSolver3D::advect_field: RK3 backtrace, trilinear sample of a
        field of spacing fh (h/2 for the density/temperature grids); a second
        field on the same grid shares the backtrace."""
        fnz, fny, fnx = field.shape
        out = torch.empty_like(field) if out is None else out
        if field2 is not None and out2 is None:
            out2 = torch.empty_like(field2)
        self._check(self.lib.vflip_advect_rk3_linear2(self.ctx, ni, nj, nk, float(h), float(dt), _p(u), _p(v), _p(w),
                                                      fnx, fny, fnz, float(fh), float(offsets[0]), float(offsets[1]),
                                                      float(offsets[2]), _p(field), _p(out),
                                                      _p(field2) if field2 is not None else None,
                                                      _p(out2) if field2 is not None else None))
        return out if field2 is None else (out, out2)

    def gen_heat(self, rho, temp, fh, dt, dens_decay, temp_decay, centre, radius, dens, heat):
        """SmokeSolver3D::gen_heat, in place on the density/temperature grids."""
        fnz, fny, fnx = rho.shape
        self._check(self.lib.vflip_gen_heat(self.ctx, fnx, fny, fnz, float(fh), float(dt), float(dens_decay),
                                            float(temp_decay), float(centre[0]), float(centre[1]), float(centre[2]),
                                            float(radius), float(dens), float(heat), _p(rho), _p(temp)))

    def add_smokeforce(self, particles, rho, temp, fh, alpha, beta, dt):
        """SmokeSolver3D::add_smokeforce, in place on the particles."""
        fnz, fny, fnx = rho.shape
        self._check(self.lib.vflip_add_smokeforce(self.ctx, _p(particles), self._np(particles), fnx, fny, fnz,
                                                  float(fh), _p(rho), _p(temp), float(alpha), float(beta), float(dt)))

    # ------------------------------------------------------------- nested subdomain
    def sub_particle_cells(self, ni, nj, nk, h, bmin, particles):
        n = self._np(particles)
        out = self._empty((n,), torch.int32)
        self._check(self.lib.vflip_sub_particle_cells(self.ctx, ni, nj, nk, float(h), *(float(b) for b in bmin),
                                                      _p(particles), n, _p(out)))
        return out

    def sub_particle_to_grid(self, ni, nj, nk, h, bmin, particles, components=(0, 1, 2)):
        """SubDomainSolver::particle_to_grid: {comp: (field, coef)} on the subdomain's face grids."""
        n = self._np(particles)
        shapes = _face_shapes(ni, nj, nk)
        outs = {c: (self._empty(shapes[c], torch.float32), self._empty(shapes[c], torch.float32)) for c in components}
        ptrs = []
        for c in range(3):
            ptrs += [_p(outs[c][0]), _p(outs[c][1])] if c in outs else [None, None]
        self._check(self.lib.vflip_sub_p2g(self.ctx, ni, nj, nk, float(h), *(float(b) for b in bmin), _p(particles),
                                           n, *ptrs))
        return outs

    def sub_particle_from_grid(self, ni, nj, nk, h, bmin, particles, du, dv, dw):
        """SubDomainSolver::particle_from_grid, in place."""
        self._check(self.lib.vflip_sub_g2p(self.ctx, ni, nj, nk, float(h), *(float(b) for b in bmin), _p(particles),
                                           self._np(particles), _p(du), _p(dv), _p(dw)))

    def sub_reorder_flip(self, ni, nj, nk, h, bmin, particles, u, v, w, nodal_phi, seed=0, capacity=None):
        """SubDomainSolver::hash_FLIP + reorder_FLIP: a new particle tensor."""
        n = self._np(particles)
        cap = 9 * ni * nj * nk if capacity is None else int(capacity)
        out = torch.empty(max(cap, 1) * PARTICLE_BYTES, dtype=torch.uint8, device=self.device)
        cnt = C.c_int()
        self._check(self.lib.vflip_sub_reorder_flip(self.ctx, ni, nj, nk, float(h), *(float(b) for b in bmin),
                                                    _p(particles), n, _p(u), _p(v), _p(w), _p(nodal_phi),
                                                    int(seed) & 0xFFFFFFFF, _p(out), cap, C.byref(cnt)))
        return out[:cnt.value * PARTICLE_BYTES]

    # ------------------------------------------------------------- main grid with its subdomain active
    @staticmethod
    def subdomain(dims, h, bmin, u, v, w, nodal_phi):
        """The nested subdomain the *_nested calls take: dims cells of spacing h
        at bmin, its face velocities and nodal solid phi (device tensors, kept
        referenced by the returned object)."""
        ni, nj, nk = (int(x) for x in dims)
        d = SubdomainC(ni, nj, nk, float(h), (C.c_float * 3)(*(float(b) for b in bmin)), _p(u), _p(v), _p(w),
                       _p(nodal_phi))
        d._tensors = (u, v, w, nodal_phi)
        return d

    def advect_flip_nested(self, ni, nj, nk, h, particles, u, v, w, nodal_phi, dt, sub):
        """advect_FLIP through the main grid's samplers with its subdomain active."""
        n = self._np(particles)
        self._check(self.lib.vflip_advect_flip_nested(self.ctx, ni, nj, nk, float(h), _p(particles), n, _p(u), _p(v),
                                                      _p(w), _p(nodal_phi), float(dt), C.byref(sub)))
        return particles

    def reorder_flip_nested(self, ni, nj, nk, h, particles, u, v, w, nodal_phi, sub, seed=0, capacity=None):
        """reorder_FLIP of the main grid with the nested solid filter: a new particle tensor."""
        n = self._np(particles)
        cap = 9 * ni * nj * nk if capacity is None else int(capacity)
        out = torch.empty(max(cap, 1) * PARTICLE_BYTES, dtype=torch.uint8, device=self.device)
        cnt = C.c_int()
        self._check(self.lib.vflip_reorder_flip_nested(self.ctx, ni, nj, nk, float(h), _p(particles), n, _p(u),
                                                       _p(v), _p(w), _p(nodal_phi), int(seed) & 0xFFFFFFFF, _p(out),
                                                       cap, C.byref(cnt), C.byref(sub)))
        return out[:cnt.value * PARTICLE_BYTES]

    def halo_select(self, particles, h, sub, capacity=None):
        """The particles inside the subdomain's box widened by half a main cell
        (h = main spacing): a new particle tensor."""
        n = self._np(particles)
        cap = n if capacity is None else int(capacity)
        out = torch.empty(max(cap, 1) * PARTICLE_BYTES, dtype=torch.uint8, device=self.device)
        cnt = C.c_int()
        self._check(self.lib.vflip_halo_select(self.ctx, _p(particles) if n else None, n, float(h), C.byref(sub),
                                               _p(out), cap, C.byref(cnt)))
        return out[:cnt.value * PARTICLE_BYTES]

    def advect_tracers_nested(self, ni, nj, nk, h, tracers, u, v, w, nodal_phi, dt, dens_decay, sub):
        """advect_tracers with the subdomain active, in place on (n, 4) float32 tracers."""
        self._check(self.lib.vflip_advect_tracers_nested(self.ctx, ni, nj, nk, float(h), _p(tracers),
                                                         tracers.shape[0], _p(u), _p(v), _p(w), _p(nodal_phi),
                                                         float(dt), float(dens_decay), C.byref(sub)))

    def emit_tracers_nested(self, tracers, h, lengths, centre, radius, count, dims, nodal_phi, sub, seed=0,
                            capacity=None):
        """emit_tracers with the subdomain's seeding: a new (m, 4) float32 tensor."""
        n = tracers.shape[0] if tracers is not None else 0
        cap = n + int(count) + 4 * sub.ni * sub.nj * sub.nk if capacity is None else int(capacity)
        out = self._empty((max(cap, 1), 4), torch.float32)
        m = C.c_int()
        self._check(self.lib.vflip_emit_tracers_nested(
            self.ctx, _p(tracers) if n else None, n, float(h), float(lengths[0]), float(lengths[1]),
            float(lengths[2]), float(centre[0]), float(centre[1]), float(centre[2]), float(radius), int(count),
            int(seed) & 0xFFFFFFFF, int(dims[0]), int(dims[1]), int(dims[2]), _p(nodal_phi), C.byref(sub), _p(out),
            cap, C.byref(m)))
        return out[:m.value]

    # ------------------------------------------------------------- tracers
    def emit_tracers(self, tracers, h, lengths, centre, radius, count, seed=0, capacity=None):
        """SmokeSolver3D::emit_tracers: returns a new (m, 4) float32 tensor."""
        n = tracers.shape[0] if tracers is not None else 0
        cap = n + int(count) if capacity is None else int(capacity)
        out = self._empty((max(cap, 1), 4), torch.float32)
        m = C.c_int()
        self._check(self.lib.vflip_emit_tracers(self.ctx, _p(tracers) if n else None, n, float(h), float(lengths[0]),
                                                float(lengths[1]), float(lengths[2]), float(centre[0]),
                                                float(centre[1]), float(centre[2]), float(radius), int(count),
                                                int(seed) & 0xFFFFFFFF, _p(out), cap, C.byref(m)))
        return out[:m.value]

    def advect_tracers(self, ni, nj, nk, h, tracers, u, v, w, nodal_phi, dt, dens_decay=0.0):
        """SmokeSolver3D::advect_tracers, in place on (n, 4) float32 tracers."""
        self._check(self.lib.vflip_advect_tracers(self.ctx, ni, nj, nk, float(h), _p(tracers), tracers.shape[0], _p(u),
                                                  _p(v), _p(w), _p(nodal_phi), float(dt), float(dens_decay)))

    def write_tracers(self, tracers, lx, directory, frame):
        """SmokeSolver3D::write_tracers: <directory>/Particle_data%04d.bin."""
        n = tracers.shape[0]
        self._check(self.lib.vflip_write_tracers(self.ctx, _p(tracers) if n else None, n, float(lx),
                                                 str(directory).encode(), int(frame)))

    def delta(self, after, before, out=None):
        if out is None:
            out = torch.empty_like(after)
        self._check(self.lib.vflip_delta(self.ctx, after.numel(), _p(after), _p(before), _p(out)))
        return out

    # ------------------------------------------------------------- FLIP
    @staticmethod
    def _np(particles):
        nbytes = particles.numel() * particles.element_size()
        if nbytes % PARTICLE_BYTES:
            raise ValueError("particle buffer is not a whole number of 40-byte records")
        return nbytes // PARTICLE_BYTES

    def particle_cells(self, ni, nj, nk, h, particles):
        n = self._np(particles)
        out = self._empty((n,), torch.int32)
        self._check(self.lib.vflip_particle_cells(self.ctx, ni, nj, nk, float(h), _p(particles), n, _p(out)))
        return out

    def particle_to_grid(self, ni, nj, nk, h, particles, components=(0, 1, 2)):
        """Returns {comp: (field, coef)} on the u/v/w face grids."""
        n = self._np(particles)
        shapes = _face_shapes(ni, nj, nk)
        outs = {c: (self._empty(shapes[c], torch.float32), self._empty(shapes[c], torch.float32)) for c in components}
        ptrs = []
        for c in range(3):
            ptrs += [_p(outs[c][0]), _p(outs[c][1])] if c in outs else [None, None]
        self._check(self.lib.vflip_p2g(self.ctx, ni, nj, nk, float(h), _p(particles), n, *ptrs))
        return outs

    def particle_from_grid(self, ni, nj, nk, h, particles, du, dv, dw, un=None, vn=None, wn=None, flip_ratio=1.0):
        n = self._np(particles)
        self._check(self.lib.vflip_g2p(self.ctx, ni, nj, nk, float(h), _p(particles), n, _p(du), _p(dv), _p(dw),
                                       _p(un), _p(vn), _p(wn), float(flip_ratio)))
        return particles

    def advect_flip(self, ni, nj, nk, h, particles, u, v, w, nodal_phi, dt):
        """SmokeSolver3D::advect_FLIP: RK3 + solid push-out, positions in place."""
        n = self._np(particles)
        self._check(self.lib.vflip_advect_flip(self.ctx, ni, nj, nk, float(h), _p(particles), n, _p(u), _p(v), _p(w),
                                               _p(nodal_phi), float(dt)))
        return particles

    def reorder_flip(self, ni, nj, nk, h, particles, u, v, w, nodal_phi, seed=0, capacity=None):
        """SmokeSolver3D::hash_FLIP + reorder_FLIP: returns a new particle
        tensor (uint8 records) with 8 particles per open cell (8-9 kept)."""
        n = self._np(particles)
        cap = 9 * ni * nj * nk if capacity is None else int(capacity)
        out = torch.empty(max(cap, 1) * PARTICLE_BYTES, dtype=torch.uint8, device=self.device)
        cnt = C.c_int()
        self._check(self.lib.vflip_reorder_flip(self.ctx, ni, nj, nk, float(h), _p(particles), n, _p(u), _p(v), _p(w),
                                                _p(nodal_phi), int(seed) & 0xFFFFFFFF, _p(out), cap, C.byref(cnt)))
        return out[:cnt.value * PARTICLE_BYTES]

    # ------------------------------------------------------------- plume
    def plume_sources(self, ni, nj, nk, h, dt, rho, temp, v, centre, radius, dens_value=1.0, heat_value=1.0,
                      alpha=0.1, beta=1.0):
        self._check(self.lib.vflip_plume_sources(self.ctx, ni, nj, nk, float(h), float(dt), _p(rho), _p(temp), _p(v),
                                                 float(centre[0]), float(centre[1]), float(centre[2]), float(radius),
                                                 float(dens_value), float(heat_value), float(alpha), float(beta)))

    # ------------------------------------------------------------- measurement
    def set_profiling(self, enable):
        self._check(self.lib.vflip_set_profiling(self.ctx, 1 if enable else 0))

    def profile_sweeps(self):
        """(launches, total_ms, fine cells) of the timed fine-level sweeps."""
        n = C.c_int(0)
        ms = C.c_double(0.0)
        cells = C.c_double(0.0)
        self._check(self.lib.vflip_profile_sweeps(self.ctx, C.byref(n), C.byref(ms), C.byref(cells)))
        return n.value, ms.value, cells.value

    PROF_KINDS = {"fine_sweep": 0, "spmv": 1, "update": 2, "advect_field": 3, "advect_pair": 4, "vcycle": 5,
                  "coarse": 6, "p2g_sort": 7, "p2g_gather": 8}

    def profile_kernels(self, kind):
        """(launches, total_ms) of the timed launches of one kind (PROF_KINDS)."""
        n = C.c_int(0)
        ms = C.c_double(0.0)
        self._check(self.lib.vflip_profile_kernels(self.ctx, self.PROF_KINDS[kind], C.byref(n), C.byref(ms)))
        return n.value, ms.value

    @property
    def launch_count(self):
        return int(self.lib.vflip_launch_count(self.ctx))

    # ------------------------------------------------------------- layout
    def bricks_to_linear(self, nx, ny, nz, bricked):
        out = self._empty((nz, ny, nx), torch.float32)
        self._check(self.lib.vflip_bricks_to_linear(self.ctx, nx, ny, nz, _p(bricked), _p(out)))
        return out

    def linear_to_bricks(self, nx, ny, nz, linear):
        pad = lambda n: (n + 7) // 8 * 8  # noqa: E731
        out = torch.zeros((pad(nz) * pad(ny) * pad(nx),), dtype=torch.float32, device=self.device)
        self._check(self.lib.vflip_linear_to_bricks(self.ctx, nx, ny, nz, _p(linear), _p(out)))
        return out
