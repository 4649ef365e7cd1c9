"""ctypes bindings for the oracle libraries.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package, and only to compare against.  The product package (vflip_b200)
never imports it.

Two libraries share one calling convention (linear layout, i fastest):
  * ``liboracle.so``        - this project's CPU restatement (vflip_oracle.cpp);
  * ``_ref/libvflip_ref.so`` - the reference's own code (build_ref.py), present
    only where the reference tree was available at build time;
  * ``_ref/libvflip_ref_dropin.so`` - the same code with the GPU drop-in
    (include/vflip/amgpcg_dropin.hpp) as its ivock::AMGPCGSolve.

Seven-point operators are numpy arrays of shape (7, nk, nj, ni), float64, in
the slot order diag, -x, +x, -y, +y, -z, +z.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libvflip_ref.so")
REF_DROPIN_SO = os.path.join(HERE, "_ref", "libvflip_ref_dropin.so")

PARTICLE_DTYPE = np.dtype([("pos", "<f4", (3,)), ("vel", "<f4", (3,)), ("dens", "<f4"), ("temp", "<f4"),
                           ("hash_idx", "<i4"), ("sub_hash_idx", "<i4")])
assert PARTICLE_DTYPE.itemsize == 40

_P = C.c_void_p
_I = C.c_int
_F = C.c_float
_D = C.c_double


class SubDesc(C.Structure):
    """The nested subdomain as the main solver's samplers see it (the layout of
    the C ABI's vflip_subdomain): cells, spacing, origin, face velocities and
    nodal solid phi."""
    _fields_ = [("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int), ("h", C.c_float), ("bmin", C.c_float * 3),
                ("u", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p), ("nodal_phi", C.c_void_p)]


def sub_desc(sub):
    """(SubDesc, arrays kept alive) from sub = dict(dims=(ni, nj, nk), h=, bmin=,
    u=, v=, w=, phi=) with numpy grids in the linear layout."""
    ni, nj, nk = (int(x) for x in sub["dims"])
    arrs = [np.ascontiguousarray(sub[k], np.float32) for k in ("u", "v", "w", "phi")]
    d = SubDesc(ni, nj, nk, float(sub["h"]), (C.c_float * 3)(*[float(x) for x in sub["bmin"]]),
                *[a.ctypes.data for a in arrs])
    return d, arrs


def _ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def build_oracle():
    """Compile liboracle.so (and the reference library when its tree exists)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
    subprocess.check_call(["python3", os.path.join(HERE, "build_ref.py")])


_libs = {}


def _load(path, prefix):
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    p = prefix
    if prefix == "oracle":
        getattr(lib, p + "_levels").argtypes = [_I, _I, _I, _P, _I, _P, _P]
        getattr(lib, p + "_rbgs").argtypes = [_I, _I, _I, _P, _P, _P, _I]
        getattr(lib, p + "_vcycle").argtypes = [_I, _I, _I, _P, _P, _P]
        getattr(lib, p + "_spmv").argtypes = [_I, _I, _I, _P, _P, _P]
        getattr(lib, p + "_amgpcg").argtypes = [_I, _I, _I, _P, _P, _P, _D, _I, _P, _P]
    else:
        getattr(lib, p + "_levels").argtypes = [_I, _I, _I, _P, _P, _P, _I, _P, _P]
        if hasattr(lib, p + "_rbgs"):  # absent from the drop-in build (the GPU solve replaces them)
            getattr(lib, p + "_rbgs").argtypes = [_I, _I, _I, _P, _P, _P, _P, _P, _I]
            getattr(lib, p + "_vcycle").argtypes = [_I, _I, _I, _P, _P, _P, _P, _P]
        getattr(lib, p + "_amgpcg").argtypes = [_I, _I, _I, _P, _P, _P, _P, _P, _D, _I, _P, _P]
        getattr(lib, p + "_delta").argtypes = [_I, _I, _I, _P, _P, _P]
    if prefix == "oracle":
        getattr(lib, p + "_project_subdomain").argtypes = [_I, _I, _I, _F, _F, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                                           _P, _P, _D, _I]
    else:
        getattr(lib, p + "_project_subdomain").argtypes = [_I, _I, _I, _F, _F, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                                           _P]
    getattr(lib, p + "_smoke_step").argtypes = [_I, _F, _F, _P, _P, _P, _P, _P, _P, _F, _F, _F, _F, _F, _F, _P, _P]
    getattr(lib, p + "_smoke_step").restype = C.c_double if prefix == "ref" else C.c_int
    getattr(lib, p + "_fraction_inside4").argtypes = [_I, _P, _P, _P, _P, _P]
    getattr(lib, p + "_face_weights").argtypes = [_I, _I, _I, _F, _P, _P, _P, _P]
    getattr(lib, p + "_project").argtypes = [_I, _I, _I, _F, _F, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                             _P, _P, _P, _P, _P]
    getattr(lib, p + "_advect_rk2").argtypes = [_I, _I, _I, _F, _F, _P, _P, _P, _I, _I, _I, _D, _D, _D, _P, _P]
    getattr(lib, p + "_hash").argtypes = [_I, _I, _I, _F, _P, _I, _P]
    getattr(lib, p + "_p2g").argtypes = [_I, _I, _I, _F, _P, _I, _I, _P, _P]
    getattr(lib, p + "_advect_flip").argtypes = [_I, _I, _I, _F, _P, _I, _P, _P, _P, _P, _F]
    getattr(lib, p + "_reorder_flip").argtypes = [_I, _I, _I, _F, _P, _I, _P, _P, _P, _P, C.c_uint, _P, _I]
    getattr(lib, p + "_reorder_flip").restype = _I
    getattr(lib, p + "_advect_cubic_clamp").argtypes = [_I, _I, _I, _F, _F, _P, _P, _P, _I, _I, _I, _D, _D, _D, _P,
                                                        _P]
    getattr(lib, p + "_advect_rk3").argtypes = [_I, _I, _I, _F, _F, _P, _P, _P, _I, _I, _I, _D, _D, _D, _D, _P, _P]
    getattr(lib, p + "_gen_heat").argtypes = [_I, _I, _I, _D, _F, _F, _F, _F, _F, _F, _F, _F, _F, _P, _P]
    getattr(lib, p + "_add_smokeforce").argtypes = [_P, _I, _I, _I, _I, _D, _P, _P, _F, _F, _F]
    getattr(lib, p + "_emit_tracers").argtypes = [_P, _I, _F, _F, _F, _F, _F, _F, _F, _F, _I, C.c_uint, _P, _I]
    getattr(lib, p + "_emit_tracers").restype = _I
    getattr(lib, p + "_advect_tracers").argtypes = [_I, _I, _I, _F, _P, _I, _P, _P, _P, _P, _F, _F]
    getattr(lib, p + "_sub_hash").argtypes = [_I, _I, _I, _F, _F, _F, _F, _P, _I, _P]
    getattr(lib, p + "_sub_p2g").argtypes = [_I, _I, _I, _F, _F, _F, _F, _P, _I, _I, _P, _P]
    getattr(lib, p + "_sub_g2p").argtypes = [_I, _I, _I, _F, _F, _F, _F, _P, _I, _P, _P, _P]
    getattr(lib, p + "_sub_reorder_flip").argtypes = [_I, _I, _I, _F, _F, _F, _F, _P, _I, _P, _P, _P, _P, C.c_uint,
                                                      _P, _I]
    getattr(lib, p + "_sub_reorder_flip").restype = _I
    sd = C.POINTER(SubDesc)
    getattr(lib, p + "_advect_flip_nested").argtypes = [_I, _I, _I, _F, _P, _I, _P, _P, _P, _P, _F, sd]
    getattr(lib, p + "_reorder_flip_nested").argtypes = [_I, _I, _I, _F, _P, _I, _P, _P, _P, _P, C.c_uint, _P, _I,
                                                         sd]
    getattr(lib, p + "_reorder_flip_nested").restype = _I
    getattr(lib, p + "_advect_tracers_nested").argtypes = [_I, _I, _I, _F, _P, _I, _P, _P, _P, _P, _F, _F, sd]
    getattr(lib, p + "_emit_tracers_nested").argtypes = [_P, _I, _F, _F, _F, _F, _F, _F, _F, _F, _I, C.c_uint, _I,
                                                         _I, _I, _P, sd, _P, _I]
    getattr(lib, p + "_emit_tracers_nested").restype = _I
    if prefix == "oracle":
        getattr(lib, p + "_halo_select").argtypes = [_P, _I, sd, _F, _P, _I]
    else:
        getattr(lib, p + "_halo_select").argtypes = [_P, _I, _F, sd, _P, _I]
    getattr(lib, p + "_solid_phi_nested").argtypes = [_I, _I, _I, _F, _P, sd, _P, _I, _P]
    getattr(lib, p + "_halo_select").restype = _I
    if prefix == "oracle":
        getattr(lib, p + "_tracer_records").argtypes = [_P, _I, _F, _P]
    else:
        getattr(lib, p + "_write_tracers").argtypes = [_P, _I, _F, C.c_char_p, _I]
    if prefix == "oracle":
        getattr(lib, p + "_g2p").argtypes = [_I, _I, _I, _F, _P, _I, _P, _P, _P, _P, _P, _P, _D]
        getattr(lib, p + "_delta").argtypes = [_I, _I, _I, _P, _P, _P]
    else:
        getattr(lib, p + "_g2p").argtypes = [_I, _I, _I, _F, _P, _I, _P, _P, _P]
    _libs[path] = lib
    return lib


# ---------------------------------------------------------------- conversions

def stencil_to_csr(st):
    """7-slot stencil (7, nk, nj, ni) -> CSR (rowstart, colindex, value) with
    the entries of every in-grid neighbour, columns ascending."""
    _, nk, nj, ni = st.shape
    n = ni * nj * nk
    flat = st.reshape(7, n)
    idx = np.arange(n, dtype=np.int64)
    i = idx % ni
    j = (idx // ni) % nj
    k = idx // (ni * nj)
    # column order: -z, -y, -x, diag, +x, +y, +z
    cols, vals, valid = [], [], []
    for slot, off, ok in ((5, -ni * nj, k > 0), (3, -ni, j > 0), (1, -1, i > 0), (0, 0, np.ones(n, bool)),
                          (2, 1, i < ni - 1), (4, ni, j < nj - 1), (6, ni * nj, k < nk - 1)):
        cols.append(idx + off)
        vals.append(flat[slot])
        valid.append(ok)
    cols = np.stack(cols, 1)
    vals = np.stack(vals, 1)
    valid = np.stack(valid, 1)
    counts = valid.sum(1)
    rowstart = np.zeros(n + 1, np.uint32)
    rowstart[1:] = np.cumsum(counts)
    return rowstart, cols[valid].astype(np.uint32), np.ascontiguousarray(vals[valid], dtype=np.float64)


# ---------------------------------------------------------------- solver API

class _Impl:
    def __init__(self, lib, prefix):
        self.lib = lib
        self.p = prefix

    def fn(self, name):
        return getattr(self.lib, self.p + "_" + name)

    def _op(self, st):
        st = np.ascontiguousarray(st, dtype=np.float64)
        if self.p == "oracle":
            return (_ptr(st),), st
        rs, ci, v = stencil_to_csr(st)
        return (_ptr(rs), _ptr(ci), _ptr(v)), (rs, ci, v)

    def levels(self, st, max_levels=16):
        _, nk, nj, ni = st.shape
        args, keep = self._op(st)
        dims = np.zeros(3 * max_levels, np.int32)
        # upper bound for all levels' stencil storage
        total = 0
        a, b, c = ni, nj, nk
        for _ in range(max_levels):
            total += 7 * a * b * c
            a, b, c = (a + 1) // 2, (b + 1) // 2, (c + 1) // 2
        out = np.zeros(total, np.float64)
        nl = self.fn("levels")(ni, nj, nk, *args, max_levels, _ptr(dims), _ptr(out))
        if nl < 0:
            raise RuntimeError("a level left the 7-point pattern")
        res, off = [], 0
        for l in range(nl):
            x, y, z = dims[3 * l:3 * l + 3]
            m = 7 * x * y * z
            res.append(out[off:off + m].reshape(7, z, y, x).copy())
            off += m
        return res

    def rbgs(self, st, b, x, iters):
        _, nk, nj, ni = st.shape
        args, keep = self._op(st)
        b = np.ascontiguousarray(b, np.float64)
        x = np.array(x, np.float64, copy=True, order="C")
        self.fn("rbgs")(ni, nj, nk, *args, _ptr(b), _ptr(x), iters)
        return x

    def vcycle(self, st, b):
        _, nk, nj, ni = st.shape
        args, keep = self._op(st)
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b)
        self.fn("vcycle")(ni, nj, nk, *args, _ptr(b), _ptr(x))
        return x

    def amgpcg(self, st, rhs, tol=1e-6, maxit=50):
        _, nk, nj, ni = st.shape
        args, keep = self._op(st)
        rhs = np.ascontiguousarray(rhs, np.float64)
        x = np.zeros_like(rhs)
        res = C.c_double(0)
        it = C.c_int(0)
        ok = self.fn("amgpcg")(ni, nj, nk, *args, _ptr(rhs), _ptr(x), tol, maxit, C.byref(res), C.byref(it))
        return x, bool(ok), res.value, it.value

    def fraction_inside4(self, bl, br, tl, tr):
        arrs = [np.ascontiguousarray(a, np.float32) for a in (bl, br, tl, tr)]
        out = np.zeros_like(arrs[0])
        self.fn("fraction_inside4")(arrs[0].size, *[_ptr(a) for a in arrs], _ptr(out))
        return out

    def face_weights(self, ni, nj, nk, h, phi):
        phi = np.ascontiguousarray(phi, np.float32)
        uw = np.zeros((nk, nj, ni + 1), np.float32)
        vw = np.zeros((nk, nj + 1, ni), np.float32)
        ww = np.zeros((nk + 1, nj, ni), np.float32)
        self.fn("face_weights")(ni, nj, nk, h, _ptr(phi), _ptr(uw), _ptr(vw), _ptr(ww))
        return uw, vw, ww

    def project(self, ni, nj, nk, h, U_in, phi, bdesc, us, vs, ws, u, v, w):
        phi = np.ascontiguousarray(phi, np.float32)
        bdesc = np.ascontiguousarray(bdesc, np.int8)
        us, vs, ws = [np.ascontiguousarray(a, np.float32) for a in (us, vs, ws)]
        u, v, w = [np.array(a, np.float32, copy=True, order="C") for a in (u, v, w)]
        n = ni * nj * nk
        p = np.zeros((nk, nj, ni), np.float64)
        rhs = np.zeros((nk, nj, ni), np.float64)
        st = np.zeros((7, nk, nj, ni), np.float64)
        uw = np.zeros_like(us)
        vw = np.zeros_like(vs)
        ww = np.zeros_like(ws)
        it = C.c_int(0)
        res = C.c_double(0)
        ok = self.fn("project")(ni, nj, nk, h, U_in, _ptr(phi), _ptr(bdesc), _ptr(us), _ptr(vs), _ptr(ws),
                                _ptr(u), _ptr(v), _ptr(w), _ptr(p), _ptr(rhs), _ptr(st), _ptr(uw), _ptr(vw),
                                _ptr(ww), C.byref(it), C.byref(res))
        assert n == p.size
        return dict(u=u, v=v, w=w, pressure=p, rhs=rhs, stencil=st, uw=uw, vw=vw, ww=ww, ok=bool(ok),
                    iterations=it.value, residual=res.value)

    def project_subdomain(self, ni, nj, nk, h, dt, phi, us, vs, ws, u, v, w, tol=1e-9, maxit=1000):
        """SubDomainSolver::pcg_projection (the reference library always uses
        1e-9 / 1000)."""
        phi = np.ascontiguousarray(phi, np.float32)
        us, vs, ws = [np.ascontiguousarray(a, np.float32) for a in (us, vs, ws)]
        u, v, w = [np.array(a, np.float32, copy=True, order="C") for a in (u, v, w)]
        p = np.zeros((nk, nj, ni), np.float64)
        rhs = np.zeros_like(p)
        st = np.zeros((7, nk, nj, ni), np.float64)
        if self.p == "oracle":
            it = C.c_int(0)
            res = C.c_double(0)
            ok = self.fn("project_subdomain")(ni, nj, nk, h, dt, _ptr(phi), _ptr(us), _ptr(vs), _ptr(ws), _ptr(u),
                                              _ptr(v), _ptr(w), _ptr(p), _ptr(rhs), _ptr(st), C.byref(it),
                                              C.byref(res), tol, maxit)
            extra = dict(ok=bool(ok), iterations=it.value, residual=res.value)
        else:
            self.fn("project_subdomain")(ni, nj, nk, h, dt, _ptr(phi), _ptr(us), _ptr(vs), _ptr(ws), _ptr(u), _ptr(v),
                                         _ptr(w), _ptr(p), _ptr(rhs), _ptr(st))
            extra = {}
        return dict(u=u, v=v, w=w, pressure=p, rhs=rhs, stencil=st, **extra)

    def advect_rk2(self, ni, nj, nk, h, dt, u, v, w, field, offsets):
        u, v, w, field = [np.ascontiguousarray(a, np.float32) for a in (u, v, w, field)]
        fnz, fny, fnx = field.shape
        out = np.zeros_like(field)
        self.fn("advect_rk2")(ni, nj, nk, h, dt, _ptr(u), _ptr(v), _ptr(w), fnx, fny, fnz, float(offsets[0]),
                              float(offsets[1]), float(offsets[2]), _ptr(field), _ptr(out))
        return out

    def advect_cubic_clamp(self, ni, nj, nk, h, dt, u, v, w, field, offsets):
        """SmokeSolver3D::advect_field_cubic_clamp (RK2 backtrace, clamped cubic sample)."""
        u, v, w, field = [np.ascontiguousarray(a, np.float32) for a in (u, v, w, field)]
        fnz, fny, fnx = field.shape
        out = np.zeros_like(field)
        self.fn("advect_cubic_clamp")(ni, nj, nk, h, dt, _ptr(u), _ptr(v), _ptr(w), fnx, fny, fnz,
                                      float(offsets[0]), float(offsets[1]), float(offsets[2]), _ptr(field), _ptr(out))
        return out

    def advect_rk3(self, ni, nj, nk, h, dt, u, v, w, field, fh, offsets=(0.0, 0.0, 0.0)):
        """SmokeSolver3D::advect_field (RK3 backtrace, trilinear sample) of a
        field of spacing fh (h/2 for the density/temperature grids)."""
        u, v, w, field = [np.ascontiguousarray(a, np.float32) for a in (u, v, w, field)]
        fnz, fny, fnx = field.shape
        out = np.zeros_like(field)
        self.fn("advect_rk3")(ni, nj, nk, h, dt, _ptr(u), _ptr(v), _ptr(w), fnx, fny, fnz, float(fh),
                              float(offsets[0]), float(offsets[1]), float(offsets[2]), _ptr(field), _ptr(out))
        return out

    def gen_heat(self, rho, temp, fh, dt, dens_decay, temp_decay, centre, radius, dens, heat):
        """SmokeSolver3D::gen_heat on copies; returns (rho, temp)."""
        rho = np.array(rho, np.float32, copy=True)
        temp = np.array(temp, np.float32, copy=True)
        fnz, fny, fnx = rho.shape
        self.fn("gen_heat")(fnx, fny, fnz, float(fh), dt, dens_decay, temp_decay, float(centre[0]),
                            float(centre[1]), float(centre[2]), radius, dens, heat, _ptr(rho), _ptr(temp))
        return rho, temp

    def add_smokeforce(self, particles, rho, temp, fh, alpha, beta, dt):
        """SmokeSolver3D::add_smokeforce on a copy of the particles."""
        p = np.array(particles, PARTICLE_DTYPE, copy=True)
        rho, temp = [np.ascontiguousarray(a, np.float32) for a in (rho, temp)]
        fnz, fny, fnx = rho.shape
        self.fn("add_smokeforce")(_ptr(p), len(p), fnx, fny, fnz, float(fh), _ptr(rho), _ptr(temp), alpha, beta, dt)
        return p

    def emit_tracers(self, tracers, h, lengths, centre, r, count, seed=0):
        """SmokeSolver3D::emit_tracers on float4 tracers (n, 4); returns the new (m, 4) array."""
        tr = np.ascontiguousarray(tracers, np.float32).reshape(-1, 4)
        cap = len(tr) + int(count) + 16
        out = np.zeros((cap, 4), np.float32)
        m = self.fn("emit_tracers")(_ptr(tr), len(tr), h, float(lengths[0]), float(lengths[1]), float(lengths[2]),
                                    float(centre[0]), float(centre[1]), float(centre[2]), r, int(count), int(seed),
                                    _ptr(out), cap)
        if m < 0 or m > cap:
            raise RuntimeError("tracer capacity")
        return out[:m].copy()

    def advect_tracers(self, ni, nj, nk, h, tracers, u, v, w, nodal_phi, dt, dens_decay):
        """SmokeSolver3D::advect_tracers on a copy of float4 tracers (n, 4)."""
        tr = np.array(tracers, np.float32, copy=True).reshape(-1, 4)
        u, v, w, phi = [np.ascontiguousarray(a, np.float32) for a in (u, v, w, nodal_phi)]
        self.fn("advect_tracers")(ni, nj, nk, h, _ptr(tr), len(tr), _ptr(u), _ptr(v), _ptr(w), _ptr(phi), float(dt),
                                  float(dens_decay))
        return tr

    def tracer_records(self, tracers, lx):
        """The float4 records write_tracers puts on disk (oracle)."""
        tr = np.ascontiguousarray(tracers, np.float32).reshape(-1, 4)
        out = np.zeros_like(tr)
        self.fn("tracer_records")(_ptr(tr), len(tr), float(lx), _ptr(out))
        return out

    def write_tracers(self, tracers, lx, directory, frame):
        """SmokeSolver3D::write_tracers (reference): <directory>/Particle_data%04d.bin."""
        tr = np.ascontiguousarray(tracers, np.float32).reshape(-1, 4)
        self.fn("write_tracers")(_ptr(tr), len(tr), float(lx), str(directory).encode(), int(frame))

    # nested subdomain: an ni x nj x nk grid of spacing h at bmin
    def sub_hash(self, ni, nj, nk, h, bmin, particles):
        particles = np.ascontiguousarray(particles, PARTICLE_DTYPE)
        out = np.zeros(len(particles), np.int32)
        self.fn("sub_hash")(ni, nj, nk, h, *(float(b) for b in bmin), _ptr(particles), len(particles), _ptr(out))
        return out

    def sub_p2g(self, ni, nj, nk, h, bmin, particles, comp):
        particles = np.ascontiguousarray(particles, PARTICLE_DTYPE)
        shape = (nk + (comp == 2), nj + (comp == 1), ni + (comp == 0))
        f = np.zeros(shape, np.float32)
        c = np.zeros(shape, np.float32)
        self.fn("sub_p2g")(ni, nj, nk, h, *(float(b) for b in bmin), _ptr(particles), len(particles), comp, _ptr(f),
                           _ptr(c))
        return f, c

    def sub_g2p(self, ni, nj, nk, h, bmin, particles, du, dv, dw):
        p = np.array(particles, PARTICLE_DTYPE, copy=True)
        du, dv, dw = [np.ascontiguousarray(a, np.float32) for a in (du, dv, dw)]
        self.fn("sub_g2p")(ni, nj, nk, h, *(float(b) for b in bmin), _ptr(p), len(p), _ptr(du), _ptr(dv), _ptr(dw))
        return p

    def sub_reorder_flip(self, ni, nj, nk, h, bmin, particles, u, v, w, nodal_phi, seed=0):
        p = np.ascontiguousarray(particles, PARTICLE_DTYPE)
        u, v, w, phi = [np.ascontiguousarray(a, np.float32) for a in (u, v, w, nodal_phi)]
        cap = 9 * ni * nj * nk + 16
        out = np.zeros(cap, PARTICLE_DTYPE)
        n = self.fn("sub_reorder_flip")(ni, nj, nk, h, *(float(b) for b in bmin), _ptr(p), len(p), _ptr(u), _ptr(v),
                                        _ptr(w), _ptr(phi), int(seed), _ptr(out), cap)
        if n < 0 or n > cap:
            raise RuntimeError("reorder capacity")
        return out[:n].copy()

    def hash(self, ni, nj, nk, h, particles):
        particles = np.ascontiguousarray(particles, PARTICLE_DTYPE)
        out = np.zeros(len(particles), np.int32)
        self.fn("hash")(ni, nj, nk, h, _ptr(particles), len(particles), _ptr(out))
        return out

    def p2g(self, ni, nj, nk, h, particles, comp):
        particles = np.ascontiguousarray(particles, PARTICLE_DTYPE)
        shape = (nk + (comp == 2), nj + (comp == 1), ni + (comp == 0))
        f = np.zeros(shape, np.float32)
        c = np.zeros(shape, np.float32)
        self.fn("p2g")(ni, nj, nk, h, _ptr(particles), len(particles), comp, _ptr(f), _ptr(c))
        return f, c

    def g2p(self, ni, nj, nk, h, particles, du, dv, dw, un=None, vn=None, wn=None, flip_ratio=1.0):
        p = np.array(particles, PARTICLE_DTYPE, copy=True)
        du, dv, dw = [np.ascontiguousarray(a, np.float32) for a in (du, dv, dw)]
        if self.p == "oracle":
            if un is None:
                un, vn, wn = du, dv, dw
            un, vn, wn = [np.ascontiguousarray(a, np.float32) for a in (un, vn, wn)]
            self.fn("g2p")(ni, nj, nk, h, _ptr(p), len(p), _ptr(du), _ptr(dv), _ptr(dw), _ptr(un), _ptr(vn),
                           _ptr(wn), float(flip_ratio))
        else:
            if flip_ratio != 1.0:
                raise ValueError("the reference's particle_from_grid is pure FLIP")
            self.fn("g2p")(ni, nj, nk, h, _ptr(p), len(p), _ptr(du), _ptr(dv), _ptr(dw))
        return p

    def advect_flip(self, ni, nj, nk, h, particles, u, v, w, nodal_phi, dt):
        """SmokeSolver3D::advect_FLIP (RK3 + solid push-out) on a copy."""
        p = np.array(particles, PARTICLE_DTYPE, copy=True)
        u, v, w, phi = [np.ascontiguousarray(a, np.float32) for a in (u, v, w, nodal_phi)]
        self.fn("advect_flip")(ni, nj, nk, h, _ptr(p), len(p), _ptr(u), _ptr(v), _ptr(w), _ptr(phi), float(dt))
        return p

    def reorder_flip(self, ni, nj, nk, h, particles, u, v, w, nodal_phi, seed=0):
        """SmokeSolver3D::hash_FLIP + reorder_FLIP; returns the new particle array."""
        p = np.ascontiguousarray(particles, PARTICLE_DTYPE)
        u, v, w, phi = [np.ascontiguousarray(a, np.float32) for a in (u, v, w, nodal_phi)]
        cap = 9 * ni * nj * nk + 16
        out = np.zeros(cap, PARTICLE_DTYPE)
        n = self.fn("reorder_flip")(ni, nj, nk, h, _ptr(p), len(p), _ptr(u), _ptr(v), _ptr(w), _ptr(phi), int(seed),
                                    _ptr(out), cap)
        if n < 0 or n > cap:
            raise RuntimeError("reorder capacity")
        return out[:n].copy()

    # ---- the main solver with its nested subdomain active; `sub` is the dict
    # of sub_desc (dims, h, bmin, u, v, w, phi)

    def advect_flip_nested(self, ni, nj, nk, h, particles, u, v, w, nodal_phi, dt, sub):
        """advect_FLIP through the blended get_velocity and the nested solid phi / normal, on a copy."""
        p = np.array(particles, PARTICLE_DTYPE, copy=True)
        u, v, w, phi = [np.ascontiguousarray(a, np.float32) for a in (u, v, w, nodal_phi)]
        d, _keep = sub_desc(sub)
        self.fn("advect_flip_nested")(ni, nj, nk, h, _ptr(p), len(p), _ptr(u), _ptr(v), _ptr(w), _ptr(phi),
                                      float(dt), C.byref(d))
        return p

    def reorder_flip_nested(self, ni, nj, nk, h, particles, u, v, w, nodal_phi, sub, seed=0):
        """hash_FLIP + reorder_FLIP of the main grid with the nested solid phi in the final filter."""
        p = np.ascontiguousarray(particles, PARTICLE_DTYPE)
        u, v, w, phi = [np.ascontiguousarray(a, np.float32) for a in (u, v, w, nodal_phi)]
        d, _keep = sub_desc(sub)
        cap = 9 * ni * nj * nk + 16
        out = np.zeros(cap, PARTICLE_DTYPE)
        n = self.fn("reorder_flip_nested")(ni, nj, nk, h, _ptr(p), len(p), _ptr(u), _ptr(v), _ptr(w), _ptr(phi),
                                           int(seed), _ptr(out), cap, C.byref(d))
        if n < 0 or n > cap:
            raise RuntimeError("reorder capacity")
        return out[:n].copy()

    def advect_tracers_nested(self, ni, nj, nk, h, tracers, u, v, w, nodal_phi, dt, dens_decay, sub):
        """advect_tracers with the subdomain active, on a copy of float4 tracers (n, 4)."""
        tr = np.array(tracers, np.float32, copy=True).reshape(-1, 4)
        u, v, w, phi = [np.ascontiguousarray(a, np.float32) for a in (u, v, w, nodal_phi)]
        d, _keep = sub_desc(sub)
        self.fn("advect_tracers_nested")(ni, nj, nk, h, _ptr(tr), len(tr), _ptr(u), _ptr(v), _ptr(w), _ptr(phi),
                                         float(dt), float(dens_decay), C.byref(d))
        return tr

    def emit_tracers_nested(self, tracers, h, lengths, centre, r, count, dims, nodal_phi, sub, seed=0):
        """emit_tracers with the subdomain's seeding (main grid dims and nodal phi); new (m, 4) array."""
        tr = np.ascontiguousarray(tracers, np.float32).reshape(-1, 4)
        phi = np.ascontiguousarray(nodal_phi, np.float32)
        d, _keep = sub_desc(sub)
        sni, snj, snk = sub["dims"]
        cap = len(tr) + int(count) + 4 * sni * snj * snk + 16
        out = np.zeros((cap, 4), np.float32)
        m = self.fn("emit_tracers_nested")(_ptr(tr), len(tr), h, float(lengths[0]), float(lengths[1]),
                                           float(lengths[2]), float(centre[0]), float(centre[1]), float(centre[2]), r,
                                           int(count), int(seed), int(dims[0]), int(dims[1]), int(dims[2]),
                                           _ptr(phi), C.byref(d), _ptr(out), cap)
        if m < 0 or m > cap:
            raise RuntimeError("tracer capacity")
        return out[:m].copy()

    def solid_phi_nested(self, ni, nj, nk, h, nodal_phi, sub, pos):
        """get_solid_phi with the subdomain active at positions (n, 3)."""
        x = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        phi = np.ascontiguousarray(nodal_phi, np.float32)
        d, _keep = sub_desc(sub)
        out = np.zeros(len(x), np.float32)
        self.fn("solid_phi_nested")(ni, nj, nk, h, _ptr(phi), C.byref(d), _ptr(x), len(x), _ptr(out))
        return out

    def halo_select(self, particles, h, sub):
        """The particles inside the subdomain box widened by half a main cell (h = main spacing)."""
        p = np.ascontiguousarray(particles, PARTICLE_DTYPE)
        d, _keep = sub_desc(sub)
        out = np.zeros(max(len(p), 1), PARTICLE_DTYPE)
        if self.p == "oracle":
            n = self.fn("halo_select")(_ptr(p), len(p), C.byref(d), float(np.float32(0.5 * float(np.float32(h)))),
                                       _ptr(out), len(out))
        else:
            n = self.fn("halo_select")(_ptr(p), len(p), float(h), C.byref(d), _ptr(out), len(out))
        if n < 0:
            raise RuntimeError("halo capacity")
        return out[:n].copy()

    def smoke_step(self, n, h, dt, phi, state, source_centre=(0.5, 0.1, 0.5), source_radius=0.1, alpha=0.1,
                   beta=1.0):
        """One grid plume step on numpy state {u, v, w, rho, temp} (updated in
        place).  Returns the library's return value: the solver's bool for
        the oracle, the seconds spent in reference code for the reference."""
        phi = np.ascontiguousarray(phi, np.float32)
        for k in ("u", "v", "w", "rho", "temp"):
            assert state[k].dtype == np.float32 and state[k].flags.c_contiguous
        it = C.c_int(0)
        res = C.c_double(0)
        r = self.fn("smoke_step")(n, float(h), float(dt), _ptr(phi), _ptr(state["u"]), _ptr(state["v"]),
                                  _ptr(state["w"]), _ptr(state["rho"]), _ptr(state["temp"]),
                                  float(source_centre[0]), float(source_centre[1]), float(source_centre[2]),
                                  float(source_radius), float(alpha), float(beta), C.byref(it), C.byref(res))
        return r, it.value, res.value

    def delta(self, after, before):
        after, before = [np.ascontiguousarray(a, np.float32) for a in (after, before)]
        out = np.zeros_like(after)
        nz, ny, nx = after.shape
        self.fn("delta")(nx, ny, nz, _ptr(after), _ptr(before), _ptr(out))
        return out


def oracle():
    """The CPU restatement (always available once built)."""
    lib = _load(ORACLE_SO, "oracle")
    if lib is None:
        raise FileNotFoundError(f"{ORACLE_SO} missing: run `make -C oracle liboracle.so`")
    return _Impl(lib, "oracle")


def reference():
    """The reference's own code, or None when it was not built here."""
    lib = _load(REF_SO, "ref")
    return None if lib is None else _Impl(lib, "ref")


def reference_dropin():
    """The reference's own code with include/vflip/amgpcg_dropin.hpp as its
    AMGPCGSolve (pressure solves on the GPU), or None when it was not built."""
    lib = _load(REF_DROPIN_SO, "ref")
    return None if lib is None else _Impl(lib, "ref")
