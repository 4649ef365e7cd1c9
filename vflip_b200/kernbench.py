"""Micro-benchmarks of the transfer kernels on seeded synthetic inputs.

    python -m vflip_b200.kernbench [--n 256] [--what advect,p2g,g2p] [--reps 5]

Times each kernel with CUDA events on the library's stream (torch's current
stream) after a warm-up and prints one JSON line per kernel with the
algorithmic bytes and GB/s:
  advect   RK2 backtrace + trilinear of one face field (u) and of the fused
           density/temperature pair, n^3 grid;
  p2g      sort-by-cell P2G of 8 jittered particles per cell on an n^3 grid
           (all three components, sort included);
  g2p      FLIP update of the same particles.
"""
import argparse
import json

import numpy as np
import torch

from . import scenes
from .solver import Solver


def timed(fn, reps):
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--what", default="advect,p2g,g2p")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--ppc", type=int, default=8)
    a = ap.parse_args()
    n, dev = a.n, "cuda:0"
    h = np.float32(1.0 / n)
    rng = np.random.default_rng(0)
    T = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)  # noqa: E731
    u, v, w = (T(x) for x in scenes.random_velocity(n, n, n, rng, scale=1.0))
    what = a.what.split(",")
    with Solver(precision=1) as s:
        if "advect" in what:
            out = torch.empty_like(u)
            ms = timed(lambda: s.advect_rk2_linear(n, n, n, h, 0.01, u, v, w, u, (0.5, 0, 0), out=out), a.reps)
            nodes = u.numel()
            print(json.dumps({"kernel": "advect_rk2 (u faces)", "n": n, "ms": ms, "nodes": nodes,
                              "alg_bytes": 8 * nodes, "GBs": 8 * nodes / ms / 1e6}))
            rho = T(rng.standard_normal((n, n, n)).astype(np.float32))
            tmp = T(rng.standard_normal((n, n, n)).astype(np.float32))
            o1, o2 = torch.empty_like(rho), torch.empty_like(tmp)
            ms = timed(lambda: s.advect_rk2_linear2(n, n, n, h, 0.01, u, v, w, rho, tmp, (0, 0, 0), out=o1, out2=o2),
                       a.reps)
            nodes = rho.numel()
            print(json.dumps({"kernel": "advect_rk2 (rho+T pair)", "n": n, "ms": ms, "nodes": nodes,
                              "alg_bytes": 16 * nodes, "GBs": 16 * nodes / ms / 1e6}))
        if "p2g" in what or "g2p" in what:
            p = scenes.jittered_particles(n, n, n, h, a.ppc, rng)
            p["vel"] = rng.standard_normal((len(p), 3)).astype(np.float32)
            rng.shuffle(p)
            parts = T(p.view(np.uint8))
            npart = len(p)
            if "p2g" in what:
                ms = timed(lambda: s.particle_to_grid(n, n, n, h, parts), a.reps)
                cells = n ** 3
                alg = npart * 24 + 3 * 8 * cells
                print(json.dumps({"kernel": "p2g (3 components, sort included)", "n": n, "particles": npart,
                                  "ms": ms, "alg_bytes": alg, "GBs": alg / ms / 1e6,
                                  "particles_per_s": npart / ms * 1e3}))
            if "g2p" in what:
                du, dv, dw = (T(x) for x in scenes.random_velocity(n, n, n, rng, scale=0.1))
                ms = timed(lambda: s.particle_from_grid(n, n, n, h, parts, du, dv, dw), a.reps)
                alg = npart * 24 + 12 * n ** 3
                print(json.dumps({"kernel": "g2p (FLIP)", "n": n, "particles": npart, "ms": ms, "alg_bytes": alg,
                                  "GBs": alg / ms / 1e6, "particles_per_s": npart / ms * 1e3}))


if __name__ == "__main__":
    main()
