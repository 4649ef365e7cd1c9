"""Autotuners: the smoother kernel and its tile shape, and the persistent
batched solve's work items.

    python -m vflip_b200.tune [--n 256] [--out vflip_b200/tuning.json]

Batched solves (VFLIP_BATCH_PERSISTENT): tune_batch times the persistent
kernel on a batch under each (cells per work item, CTAs per SM) candidate and
records the fastest per batch signature (precision + sorted sides) in a JSON
cache (BATCH_CACHE, or $VFLIP_BATCH_TUNE); tuned_batch_kwargs returns the
recorded choice as Solver keyword arguments.

For one grid size it times plain-FP32 MGPCG solves of the plume operator
(box walls + sphere obstacle) under each candidate - smoother kernel
(0 automatic, 2 3-D-tiled TMA, 3 full-row TMA with register carry, 4 full-row TMA without it), copy groups in flight, output rows per
tile (full-row kernel), plane ranges per launch, resident CTAs per SM,
threads per CTA, planes prefetched into L2 - reading the fine-level smoother's launch times from the
library's own CUDA events (vflip_set_profiling), and records the fastest
shape per grid size in a JSON cache (tuned_kwargs turns an entry into Solver
keyword arguments; the library's automatic choice is what the measurements
below selected as its default).
"""
import argparse
import json
import os

import numpy as np
import torch

from . import scenes
from .solver import Solver

HERE = os.path.dirname(os.path.abspath(__file__))
CACHE = os.path.join(HERE, "tuning.json")

# (kernel, depth, tile rows, plane ranges, CTAs per SM, threads per CTA,
# L2 prefetch planes); 0 = the library's choice, prefetch -1 = none
CANDIDATES = [
    (3, 1, 0, 0, 1, 0, -1), (3, 1, 0, 0, 1, 0, 2), (3, 1, 0, 0, 1, 0, 4), (3, 2, 0, 0, 1, 0, 2),
    (4, 1, 0, 0, 1, 512, -1), (4, 1, 0, 0, 1, 512, 2), (4, 1, 0, 0, 1, 576, 2), (4, 2, 0, 0, 1, 0, 2),
    (4, 2, 5, 3, 1, 0, 0), (4, 1, 2, 0, 2, 0, 0), (2, 1, 0, 0, 0, 0, 0), (2, 2, 0, 0, 0, 0, 0), (2, 2, 0, 4, 0, 0, 0),
]


def _shape7(shape):
    """Cached shapes from before the thread count and the prefetch were knobs
    have 4 to 6 entries."""
    shape = list(shape)
    if len(shape) == 4:
        shape = [0] + shape
    return shape + [0] * (7 - len(shape))


def load_cache():
    if os.path.exists(CACHE):
        with open(CACHE) as f:
            return json.load(f)
    return {}


def tuned_kwargs(n):
    """Solver keyword arguments recorded for an n^3 grid (empty if none)."""
    entry = load_cache().get(str(n))
    if not entry:
        return {}
    k, d, t, r, c, th, pf = _shape7(entry["shape"])
    return dict(sweep_kernel=k, smoother_depth=d, smoother_tile_rows=t, smoother_plane_ranges=r,
                smoother_ctas_per_sm=c, smoother_threads=th, smoother_prefetch=pf)


def problem(n, dev):
    h = np.float32(1.0 / n)
    phi = np.minimum(scenes.box_walls_phi(n, n, n, h), scenes.sphere_phi(n, n, n, h, (0.5, 0.5, 0.5), 0.15))
    rng = np.random.default_rng(0)
    u, v, w = scenes.random_velocity(n, n, n, rng)
    zs = [np.zeros(s, np.float32) for s in scenes.face_shapes(n, n, n)]
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    with Solver(precision=1) as s:
        st, rhs = s.assemble(n, n, n, h, 0.0, T(phi), T(np.zeros((n, n, n), np.int8)), T(zs[0]), T(zs[1]),
                             T(zs[2]), T(u), T(v), T(w))
    return st, rhs


def measure(st, rhs, shape, reps=2, precision=1):
    k, d, t, r, c, th, pf = _shape7(shape)
    with Solver(precision=precision, sweep_kernel=k, smoother_depth=d, smoother_tile_rows=t,
                smoother_plane_ranges=r, smoother_ctas_per_sm=c, smoother_threads=th,
                smoother_prefetch=pf) as s:
        s.amgpcg_solve(st, rhs, 1e-6, 50)  # warm (allocations)
        s.set_profiling(True)
        s.profile_sweeps()
        tot = 0.0
        for _ in range(reps):
            ok, _, stats = s.amgpcg_solve(st, rhs, 1e-6, 50)
            tot += stats.solve_ms
        nl, ms, cells = s.profile_sweeps()
        s.set_profiling(False)
    return {"shape": list(shape), "sweep_ms": ms / max(nl, 1), "solve_ms": tot / reps, "sweeps": nl,
            "gbs": 28 * cells / (ms / max(nl, 1)) / 1e6 if nl else None}


BATCH_CACHE = os.environ.get("VFLIP_BATCH_TUNE", os.path.join(HERE, "batch_tuning.json"))
BATCH_CANDIDATES = [(chunk, ctas) for chunk in (4096, 8192, 16384, 32768, 65536) for ctas in (0, 1, 2)]


def batch_key(precision, sides):
    return f"p{int(precision)}:" + ",".join(str(int(x)) for x in sorted(sides))


def load_batch_cache(path=None):
    path = path or BATCH_CACHE
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def tuned_batch_kwargs(precision, sides, path=None):
    """Solver keyword arguments recorded for this batch signature (empty if none)."""
    e = load_batch_cache(path).get(batch_key(precision, sides))
    return dict(batch_chunk=e["chunk"], batch_ctas_per_sm=e["ctas_per_sm"]) if e else {}


def tune_batch(systems, sides, precision=1, tol=1e-6, maxit=100, reps=1, candidates=None, path=None):
    """Times VFLIP_BATCH_PERSISTENT on `systems` (the (stencil, rhs) device
    pairs of Solver.batched_solve) under each (chunk, CTAs per SM)
    candidate - the whole call, hierarchy set-up included, best of `reps`
    after one untimed call - and records the fastest for this batch's
    signature in the JSON cache.  Returns (best entry, all measurements)."""
    rows = []
    for chunk, ctas in candidates or BATCH_CANDIDATES:
        with Solver(precision=precision, batch_chunk=chunk, batch_ctas_per_sm=ctas) as s:
            ok, _, st = s.batched_solve(systems, tol, maxit, mode=2)
            best = None
            for _ in range(reps):
                ok, _, st = s.batched_solve(systems, tol, maxit, mode=2)
                ms = st[0].solve_ms if st else 0.0
                best = ms if best is None else min(best, ms)
            rows.append({"chunk": chunk, "ctas_per_sm": ctas, "ms": best, "kernel_ms": s.last_ms,
                         "converged": bool(ok)})
    good = [r for r in rows if r["converged"]]
    if not good:
        return None, rows
    best = min(good, key=lambda r: r["ms"])
    path = path or BATCH_CACHE
    cache = load_batch_cache(path)
    cache[batch_key(precision, sides)] = best
    try:
        with open(path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    except OSError:  # a read-only install keeps the choice for this call only
        pass
    return best, rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--out", default=CACHE)
    ap.add_argument("--solve-once", action="store_true",
                    help="assemble the operator and run one FP32 solve (a small target for profilers)")
    ap.add_argument("--precision", type=int, default=1)
    ap.add_argument("--sweep-kernel", type=int, default=0, help="smoother kernel of --solve-once")
    ap.add_argument("--only-kernel", type=int, default=None, help="tune only the candidates of this smoother kernel")
    a = ap.parse_args()
    st, rhs = problem(a.n, "cuda:0")
    if a.solve_once:
        with Solver(precision=a.precision, sweep_kernel=a.sweep_kernel) as s:
            ok, _, stats = s.amgpcg_solve(st, rhs, 1e-6, 50)
        print(json.dumps({"n": a.n, "converged": ok, "iterations": stats.iterations, "solve_ms": stats.solve_ms}))
        return
    results = []
    for shape in CANDIDATES:
        if a.only_kernel is not None and shape[0] != a.only_kernel:
            continue
        try:
            r = measure(st, rhs, shape)
        except Exception as e:  # a shape the library rejects
            r = {"shape": list(shape), "error": str(e)}
        results.append(r)
        print(json.dumps(r), flush=True)
    ok = [r for r in results if "sweep_ms" in r]
    best = min(ok, key=lambda r: r["solve_ms"])
    cache = load_cache()
    cache[str(a.n)] = {"shape": best["shape"], "sweep_ms": best["sweep_ms"], "solve_ms": best["solve_ms"]}
    with open(a.out, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    print("best", json.dumps(best))


if __name__ == "__main__":
    main()
