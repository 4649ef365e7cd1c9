#!/usr/bin/env python3
"""Generates the golden fixtures in this directory by running the
reference's OWN code (oracle/_ref/libvflip_ref.so, compiled from the vFLIP
sources by oracle/build_ref.py) on small seeded inputs.

    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py smoke      # only smoke.npz (likewise tracers)

Each fixture (.npz) stores its inputs and the reference's outputs, so the
tests need neither the reference tree nor its library: they check the
oracle restatement (CPU) and the CUDA library (GPU) against these arrays.
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from vflip_b200 import scenes  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def make_smoke(R):
    """The grid advection forms of SmokeSolver3D and the smoke scalars:
    advect_field_cubic_clamp on the four grid kinds, advect_field (RK3) of
    density and temperature on the 2x grid at h/2, gen_heat, add_smokeforce."""
    rng = np.random.default_rng(31)
    ni, nj, nk = 12, 10, 9
    h = np.float32(1 / 12)  # not a power of two: exercises the true division
    dt = np.float32(0.06)
    u, v, w = scenes.random_velocity(ni, nj, nk, rng, scale=3.0)
    out = {}
    for name, offs, shape in (("u", (0.5, 0, 0), (nk, nj, ni + 1)), ("v", (0, 0.5, 0), (nk, nj + 1, ni)),
                              ("w", (0, 0, 0.5), (nk + 1, nj, ni)), ("c", (0, 0, 0), (nk, nj, ni))):
        f = rng.standard_normal(shape).astype(np.float32)
        out["cubic_in_" + name] = f
        out["cubic_out_" + name] = R.advect_cubic_clamp(ni, nj, nk, h, dt, u, v, w, f, offs)
    fh = float(h) / 2
    rho = rng.random((2 * nk, 2 * nj, 2 * ni)).astype(np.float32)
    temp = rng.random((2 * nk, 2 * nj, 2 * ni)).astype(np.float32)
    out["rk3_rho"] = R.advect_rk3(ni, nj, nk, h, dt, u, v, w, rho, fh)
    out["rk3_temp"] = R.advect_rk3(ni, nj, nk, h, dt, u, v, w, temp, fh)
    heat = dict(dt=0.06, dens_decay=0.1, temp_decay=0.3, centre=(0.5, 0.12, 0.45), radius=0.2, dens=1.0, heat=4.0)
    out["heat_rho"], out["heat_temp"] = R.gen_heat(out["rk3_rho"], out["rk3_temp"], fh, **heat)
    p = scenes.random_particles(ni, nj, nk, h, 3000, rng, margin=1.5)
    out["force_particles"] = R.add_smokeforce(p, out["heat_rho"], out["heat_temp"], fh, 0.1, 0.35, 0.06).view(np.uint8)
    np.savez_compressed(os.path.join(OUT, "smoke.npz"), dims=np.array([ni, nj, nk], np.int32), h=h, dt=dt, u=u, v=v,
                        w=w, rho=rho, temp=temp, particles=p.view(np.uint8),
                        heat_params=np.array([heat["dt"], heat["dens_decay"], heat["temp_decay"], *heat["centre"],
                                              heat["radius"], heat["dens"], heat["heat"]], np.float32),
                        force_params=np.array([0.1, 0.35, 0.06], np.float32), **out)


def make_tracers(R):
    """SmokeSolver3D tracers: emit_tracers (the kept prefix and the count;
    new positions come from rand()), advect_tracers and write_tracers' bytes."""
    import tempfile

    rng = np.random.default_rng(37)
    ni, nj, nk = 14, 12, 10
    h = np.float32(1 / 14)
    lengths = np.array([1.0, h * nj, h * nk], np.float32)
    tr = np.concatenate([rng.uniform(-0.05, 1.05, (1500, 3)), rng.uniform(0.0, 0.05, (1500, 1))], 1)
    tr = tr.astype(np.float32)
    emitted = R.emit_tracers(tr, h, lengths, (0.5, 0.2, 0.4), 0.1, 300, seed=1)
    phi = scenes.random_phi(ni, nj, nk, h, rng, n_spheres=2)
    u, v, w = scenes.random_velocity(ni, nj, nk, rng, scale=0.6)
    adv = R.advect_tracers(ni, nj, nk, h, tr, u, v, w, phi, 0.03, 0.7)
    d = tempfile.mkdtemp()
    R.write_tracers(adv, lengths[0], d, 12)
    raw = np.fromfile(os.path.join(d, "Particle_data0012.bin"), np.uint8)
    np.savez_compressed(os.path.join(OUT, "tracers.npz"), dims=np.array([ni, nj, nk], np.int32), h=h,
                        lengths=lengths, tracers=tr, emit_kept=emitted[:len(emitted) - 300], emit_count=len(emitted),
                        phi=phi, u=u, v=v, w=w, dt=np.float32(0.03), dens_decay=np.float32(0.7), advected=adv,
                        file_bytes=raw)


def make_subdomain(R):
    """The nested subdomain's particle transfers (SubDomainSolver): hash,
    widened P2G (3 components), G2P and reorder without seeding (8 particles
    per cell), on a 14 x 12 x 13 grid at h = 1/64 whose origin is off zero."""
    rng = np.random.default_rng(67)
    ni, nj, nk = 12, 10, 11
    h = np.float32(1 / 64)
    bmin = np.array([0.25, 0.3, 0.2], np.float32)
    p = scenes.random_particles(ni, nj, nk, h, 3000, rng, margin=1.5)
    p["pos"] += bmin
    out = {"cells": R.sub_hash(ni, nj, nk, h, bmin, p)}
    for c in range(3):
        out[f"p2g_f{c}"], out[f"p2g_c{c}"] = R.sub_p2g(ni, nj, nk, h, bmin, p, c)
    du, dv, dw = scenes.random_velocity(ni, nj, nk, rng)
    out["g2p"] = R.sub_g2p(ni, nj, nk, h, bmin, p, du, dv, dw).view(np.uint8)
    phi = scenes.random_phi(ni, nj, nk, h, rng, n_spheres=2)
    q = scenes.jittered_particles(ni, nj, nk, h, 8, rng)
    q["pos"] += bmin
    out["reorder"] = R.sub_reorder_flip(ni, nj, nk, h, bmin, q, du, dv, dw, phi).view(np.uint8)
    np.savez_compressed(os.path.join(OUT, "subdomain.npz"), dims=np.array([ni, nj, nk], np.int32), h=h, bmin=bmin,
                        particles=p.view(np.uint8), du=du, dv=dv, dw=dw, phi=phi, jittered=q.view(np.uint8), **out)


def make_nested(R):
    """The main solver with its nested subdomain active (SmokeSolver3D +
    SubDomainSolver coupling): advect_FLIP through the blended velocity and
    the nested solid phi/normal, reorder_FLIP without seeding (its solid
    filter reads the nested phi), the halo selection, advect_tracers, the
    nested get_solid_phi at probe points, and emit_tracers with the
    subdomain's seeding (rand(): kept part exact, seeds recorded)."""
    sc = scenes.nested_scene(seed=71, dims=(16, 14, 12), lo=(4, 3, 3), cells=(8, 7, 6))
    ni, nj, nk = sc["dims"]
    h, u, v, w, phi, sub, rng = sc["h"], sc["u"], sc["v"], sc["w"], sc["phi"], sc["sub"], sc["rng"]
    p = scenes.random_particles(ni, nj, nk, h, 4000, rng)
    out = {"advect": R.advect_flip_nested(ni, nj, nk, h, p, u, v, w, phi, 0.01, sub).view(np.uint8)}
    q = scenes.jittered_particles(ni, nj, nk, h, 8, rng)
    q = np.concatenate([q, q[rng.integers(0, len(q), 300)]])
    r = R.reorder_flip_nested(ni, nj, nk, h, q, u, v, w, phi, sub)
    out["reorder_count"] = np.int32(len(r))
    out["reorder_sha256"] = np.array(hashlib.sha256(r.tobytes()).hexdigest())
    out["halo"] = R.halo_select(p, h, sub).view(np.uint8)
    tr = np.concatenate([p["pos"], rng.uniform(0.0, 1.0, (len(p), 1)).astype(np.float32)], 1)
    out["tracers_advected"] = R.advect_tracers_nested(ni, nj, nk, h, tr, u, v, w, phi, 0.01, 0.1, sub)
    probes = rng.uniform(0.0, 1.0, (4000, 3)).astype(np.float32) * np.array([ni, nj, nk], np.float32) * h
    out["probe_phi"] = R.solid_phi_nested(ni, nj, nk, h, phi, sub, probes)
    lengths = np.array([ni, nj, nk], np.float32) * h
    e = R.emit_tracers_nested(tr, h, lengths, (0.3, 0.15, 0.25), 0.06, 400, (ni, nj, nk), phi, sub, seed=5)
    kept = R.emit_tracers(tr, h, lengths, (0.3, 0.15, 0.25), 0.06, 0, seed=5)
    sub_arrays = {"sub_" + k: np.asarray(sub[k]) for k in ("dims", "h", "bmin", "u", "v", "w", "phi")}
    np.savez_compressed(os.path.join(OUT, "nested.npz"), dims=np.array([ni, nj, nk], np.int32), h=h, u=u, v=v, w=w,
                        phi=phi, particles=p.view(np.uint8), jittered=q.view(np.uint8), tracers=tr, probes=probes,
                        emit_kept=kept, emit_seeds=e[len(kept) + 400:], emit_count=np.int32(len(e)), **sub_arrays,
                        **out)


def main(which=()):
    R = oracle.reference()
    if R is None:
        sys.exit("oracle/_ref/libvflip_ref.so is not built (python oracle/build_ref.py)")
    if which:
        if "smoke" in which:
            make_smoke(R)
        if "tracers" in which:
            make_tracers(R)
        if "subdomain" in which:
            make_subdomain(R)
        if "nested" in which:
            make_nested(R)
        return
    # 1. projection (face weights, inflow, assembly, AMGPCG 1e-6/50, gradient)
    #    on odd, non-cubic grids with inflow and moving solids
    for tag, (ni, nj, nk), seed in (("proj_a", (14, 12, 11), 11), ("proj_b", (19, 17, 23), 12)):
        pr = scenes.projection_problem(ni, nj, nk, seed=seed, inflow=True, solid_velocity=True)
        out = R.project(**pr)
        levels = R.levels(out["stencil"])
        b = out["rhs"]
        x3 = R.rbgs(out["stencil"], b, np.zeros_like(b), 3)
        vc = R.vcycle(out["stencil"], b)
        p, ok, res, it = R.amgpcg(out["stencil"], b)
        arrays = {k: v for k, v in pr.items() if isinstance(v, np.ndarray)}
        meta = np.array([ni, nj, nk], np.int32)
        np.savez_compressed(os.path.join(OUT, f"{tag}.npz"), dims=meta, h=np.float32(pr["h"]),
                            U_in=np.float32(pr["U_in"]), **{"in_" + k: v for k, v in arrays.items()},
                            out_u=out["u"], out_v=out["v"], out_w=out["w"], out_pressure=out["pressure"],
                            out_rhs=out["rhs"], out_stencil=out["stencil"], out_uw=out["uw"], out_vw=out["vw"],
                            out_ww=out["ww"], out_iterations=np.int32(out["iterations"]),
                            out_residual=np.float64(out["residual"]), rbgs3=x3, vcycle=vc, pcg_x=p,
                            pcg_ok=np.int32(ok), pcg_res=np.float64(res), pcg_it=np.int32(it),
                            n_levels=np.int32(len(levels)),
                            **{f"level{l}": lv for l, lv in enumerate(levels)})
    # 1b. the nested subdomain's projection (dt-scaled, tolerance 1e-9)
    pr = scenes.projection_problem(22, 19, 25, seed=13, solid_velocity=True)
    out = R.project_subdomain(pr["ni"], pr["nj"], pr["nk"], pr["h"], 0.005, pr["phi"], pr["us"], pr["vs"], pr["ws"],
                              pr["u"], pr["v"], pr["w"])
    np.savez_compressed(os.path.join(OUT, "proj_sub.npz"), dims=np.array([22, 19, 25], np.int32),
                        h=np.float32(pr["h"]), dt=np.float32(0.005),
                        **{"in_" + k: pr[k] for k in ("phi", "us", "vs", "ws", "u", "v", "w")},
                        **{"out_" + k: out[k] for k in ("u", "v", "w", "pressure", "rhs", "stencil")})
    # 2. multi-level hierarchy on a grid big enough for three levels
    st = scenes.uniform_laplacian(40, 37, 30)
    levels = R.levels(st)
    np.savez_compressed(os.path.join(OUT, "levels_uniform.npz"), dims=np.array([40, 37, 30], np.int32),
                        n_levels=np.int32(len(levels)), **{f"level{l}": lv for l, lv in enumerate(levels)})
    # 3. advection of the four grid kinds
    rng = np.random.default_rng(21)
    ni, nj, nk = 13, 11, 9
    h = np.float32(1 / 13)
    u, v, w = scenes.random_velocity(ni, nj, nk, rng, scale=3.0)
    fields = {}
    for name, offs, shape in (("u", (0.5, 0, 0), (nk, nj, ni + 1)), ("v", (0, 0.5, 0), (nk, nj + 1, ni)),
                              ("w", (0, 0, 0.5), (nk + 1, nj, ni)), ("c", (0, 0, 0), (nk, nj, ni))):
        f = rng.standard_normal(shape).astype(np.float32)
        fields["in_" + name] = f
        fields["out_" + name] = R.advect_rk2(ni, nj, nk, h, 0.07, u, v, w, f, offs)
    np.savez_compressed(os.path.join(OUT, "advect.npz"), dims=np.array([ni, nj, nk], np.int32), h=h,
                        dt=np.float32(0.07), u=u, v=v, w=w, **fields)
    # 4. particles: hash, P2G (3 components), G2P
    ni, nj, nk = 9, 8, 7
    h = np.float32(1 / 9)
    p = scenes.random_particles(ni, nj, nk, h, 4000, rng, margin=1.5)
    du, dv, dw = scenes.random_velocity(ni, nj, nk, rng)
    out = {"cells": R.hash(ni, nj, nk, h, p)}
    for c in range(3):
        f, cf = R.p2g(ni, nj, nk, h, p, c)
        out[f"p2g_f{c}"] = f
        out[f"p2g_c{c}"] = cf
    g = R.g2p(ni, nj, nk, h, p, du, dv, dw)
    np.savez_compressed(os.path.join(OUT, "transfer.npz"), dims=np.array([ni, nj, nk], np.int32), h=h,
                        particles=p.view(np.uint8), du=du, dv=dv, dw=dw, g2p=g.view(np.uint8), **out)
    make_smoke(R)
    make_tracers(R)
    make_subdomain(R)
    make_nested(R)
    for fn in sorted(os.listdir(OUT)):
        if fn.endswith(".npz"):
            print(fn, os.path.getsize(os.path.join(OUT, fn)))


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
