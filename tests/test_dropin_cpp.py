"""The header-only C++ drop-in (include/vflip/amgpcg_dropin.hpp): compiles
against a reference-shaped SparseMatrix (CPU) and, on a GPU, solves the
pcg_projection system like the reference solver (checked against the
oracle).  The coupled time_step sequence in C (tests/cpp/nested_step.c)
compiles as C99 and, on a GPU, steps like the Python stepper."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "dropin_main.cpp")


def build(tmp_path):
    from vflip_b200 import build as vb

    vb.build()
    exe = str(tmp_path / "dropin_main")
    libdir = os.path.join(ROOT, "vflip_b200")
    subprocess.check_call(["g++", "-O2", "-std=c++14", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                           "-L", libdir, "-l:libvflip_gpu.so", f"-Wl,-rpath,{libdir}"])
    return exe


def test_dropin_compiles(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_dropin_solves_like_the_reference(tmp_path, orc):
    pytest.importorskip("torch")
    exe = build(tmp_path)
    n = 24
    out = str(tmp_path / "out.bin")
    subprocess.check_call([exe, str(n), out])
    data = np.fromfile(out, np.float64)
    rhs, p, tail = data[:n ** 3], data[n ** 3:2 * n ** 3], data[2 * n ** 3:]
    from vflip_b200 import scenes

    h = np.float32(1.0 / n)
    o = np.ones((n + 1, n + 1, n + 1), np.float32)
    st = scenes.poisson_stencil(n, n, n, h, o[:n, :n, :n + 1], o[:n, :n + 1, :n], o[:n + 1, :n, :n])
    x, ok, res, it = orc.amgpcg(st, rhs.reshape(n, n, n))
    assert bool(tail[0]) == ok and int(tail[1]) == it
    assert np.linalg.norm(p - x.ravel()) <= 1e-11 * np.linalg.norm(x)


NESTED_SRC = os.path.join(ROOT, "tests", "cpp", "nested_step.c")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
C99 = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), "-I",
       os.path.join(CUDA_HOME, "include")]


def test_nested_step_sequence_compiles_as_c():
    """The coupled time_step sequence (C ABI + cudaMemcpyAsync,
    tests/cpp/nested_step.c) compiles as C99 against include/vflip.h with
    warnings as errors."""
    subprocess.check_call(C99 + ["-fsyntax-only", NESTED_SRC])


class GridT(C.Structure):
    _fields_ = [("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int), ("h", C.c_float), ("phi", C.c_void_p),
                ("bdesc", C.c_void_p), ("us", C.c_void_p), ("vs", C.c_void_p), ("ws", C.c_void_p)] + [
                (k, C.c_void_p) for k in ("u", "v", "w", "uc", "vc", "wc", "du", "dv", "dw", "u0", "v0", "w0",
                                          "pressure")]


EMITTER = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p)


class StepParamsT(C.Structure):
    _fields_ = [("dt", C.c_float), ("flip_ratio", C.c_double), ("seed", C.c_uint), ("tracer_count", C.c_int),
                ("src_c", C.c_float * 3), ("src_r", C.c_float), ("dens_decay", C.c_float), ("emitter", EMITTER),
                ("user", C.c_void_p), ("stream", C.c_void_p)]


@pytest.mark.gpu
def test_nested_step_sequence_steps_like_the_python_stepper(tmp_path):
    """nested_step.c's nested_flip_step, from the state after one step of
    NestedFlipSim, gives the same particles (main and subdomain), tracers and
    velocities as NestedFlipSim.step, byte for byte: the pre-projection copies,
    the emitter and the subdomain's own seed are where the Python stepper has
    them."""
    torch = pytest.importorskip("torch")
    from vflip_b200 import build as vb
    from vflip_b200.flip import NestedFlipSim, NestedParams
    from vflip_b200.particles import PARTICLE_BYTES
    from vflip_b200.solver import Solver

    vb.build()
    so = str(tmp_path / "libnested_step.so")
    libdir = os.path.join(ROOT, "vflip_b200")
    subprocess.check_call(C99 + ["-O2", "-shared", "-fPIC", NESTED_SRC, "-o", so, "-L", libdir, "-l:libvflip_gpu.so",
                                 f"-Wl,-rpath,{libdir}", "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart"])
    lib = C.CDLL(so)
    lib.nested_flip_step.restype = C.c_int
    n = 24
    prm = NestedParams(n=n, dt=0.02, source_radius=0.2, obstacle_radius=0.1, seed=4, tracers_per_step=200)
    with Solver(precision=0) as s:
        sim = NestedFlipSim(s, prm)
        sim.step()
        # the state the next step starts from (the caller appends the subdomain's particles)
        flip = torch.cat([sim.particles, sim.sub_particles])
        npart = flip.numel() // PARTICLE_BYTES
        vel = [x.clone() for x in sim.vel]
        svel = [x.clone() for x in sim.sub_vel]
        tracers = sim.tracers.clone()
        seed = prm.seed + sim.steps
        sim.step()
        want = {"p": sim.particles, "sp": sim.sub_particles, "tr": sim.tracers, "vel": sim.vel, "svel": sim.sub_vel}

        dev = s.device
        sni, snj, snk = sim.sdims

        def grid(ni, nj, nk, h, phi, bdesc, solid, u, v, w):
            t = {k: torch.empty_like(x) for k, x in zip(("uc", "vc", "wc"), (u, v, w))}
            t.update({k + s_: torch.empty_like(x) for s_ in ("0",) for k, x in zip(("u", "v", "w"), (u, v, w))})
            t.update({"d" + k: torch.empty_like(x) for k, x in zip(("u", "v", "w"), (u, v, w))})
            t["pressure"] = torch.empty((nk, nj, ni), dtype=torch.float64, device=dev)
            t.update(u=u, v=v, w=w)
            g = GridT(ni, nj, nk, float(h), phi.data_ptr(), bdesc.data_ptr() if bdesc is not None else None,
                      *(x.data_ptr() for x in solid),
                      *(t[k].data_ptr() for k in ("u", "v", "w", "uc", "vc", "wc", "du", "dv", "dw", "u0", "v0", "w0",
                                                  "pressure")))
            return g, t

        g, gt = grid(n, n, n, np.float32(prm.h), sim.phi, sim.bdesc, sim.solid, *vel)
        sgt_vel = [torch.zeros_like(x) for x in svel]
        sg, sgt = grid(sni, snj, snk, sim.sh, sim.sphi, None, sim.sub_solid, *sgt_vel)
        sub = s.subdomain(sim.sdims, sim.sh, sim.bmin, *svel, sim.sphi)

        def emit(user, v):
            gt["v"].masked_fill_(sim.source_v, prm.inflow)
            return 0

        P = StepParamsT(prm.dt, prm.flip_ratio, seed, prm.tracers_per_step, (C.c_float * 3)(*prm.source_centre),
                        prm.source_radius, prm.dens_decay, EMITTER(emit), None, s.stream.cuda_stream)
        cap2, scap2 = 9 * n ** 3, 9 * sni * snj * snk
        flip2 = torch.empty(cap2 * PARTICLE_BYTES, dtype=torch.uint8, device=dev)
        sflip = torch.empty(max(npart, 1) * PARTICLE_BYTES, dtype=torch.uint8, device=dev)
        sflip2 = torch.empty(scap2 * PARTICLE_BYTES, dtype=torch.uint8, device=dev)
        nt = tracers.shape[0]
        tcap = nt + prm.tracers_per_step + 4 * sni * snj * snk
        tracers2 = torch.empty((tcap, 4), dtype=torch.float32, device=dev)
        np_out, snp_out, nt_out = C.c_int(), C.c_int(), C.c_int()
        rc = lib.nested_flip_step(s.ctx, C.byref(P), C.byref(g), C.byref(sg), C.byref(sub), C.c_void_p(flip.data_ptr()),
                                  npart, C.c_void_p(flip2.data_ptr()), cap2, C.byref(np_out),
                                  C.c_void_p(sflip.data_ptr()), npart, C.c_void_p(sflip2.data_ptr()), scap2,
                                  C.byref(snp_out), C.c_void_p(tracers.data_ptr()) if nt else None, nt,
                                  C.c_void_p(tracers2.data_ptr()), tcap, C.byref(nt_out))
        torch.cuda.synchronize()
        assert rc == 0
        assert torch.equal(flip2[:np_out.value * PARTICLE_BYTES], want["p"])
        assert torch.equal(sflip2[:snp_out.value * PARTICLE_BYTES], want["sp"])
        assert torch.equal(tracers2[:nt_out.value], want["tr"])
        for a, b in zip((gt["u"], gt["v"], gt["w"]), want["vel"]):
            assert torch.equal(a, b)
        for a, b in zip((sgt["u"], sgt["v"], sgt["w"]), want["svel"]):
            assert torch.equal(a, b)
