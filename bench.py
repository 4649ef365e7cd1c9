#!/usr/bin/env python3
"""Benchmark of the vFLIP hot path on B200: steps/s of the 256^3 smoke plume.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--n 256]
                    [--precision fp32|fp64|mixed] [--no-cpu-baseline]

A step (the unit of the metric) is one smoke-plume step on a 256^3 MAC grid
with the centred sphere obstacle and box walls: RK2 semi-Lagrangian
trilinear advection of u, v, w, density and temperature, the density /
temperature source and buoyancy, and the pressure projection with plain
MGPCG (V(4,4) red-black Gauss-Seidel, Galerkin coarsening, 200 coarsest
sweeps) to |r|_inf <= 1e-6 |rhs|_inf, i.e. SmokeSolver3D::pcg_projection's
solve.  Synthetic seeded state; the grid fields (335 MB) are larger than L2,
so no L2 flush is needed between steps.

Multi-GPU: the path does not shard - every rank runs an independent replica
on its own GPU ("replicas only", weak scaling); value is the sum of the
replicas' steps/s (N * K / max-over-ranks time).

--impl reference times the reference's own CPU code (oracle/_ref, compiled
from the vFLIP sources: SubDomainSolver::advect_field + pcg_projection) on
the same workload on this box's host cores; when that library is absent it
times the oracle restatement (kind "port").
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "256³ steps/s @1e-6 residual, learned-precond vs plain MGPCG; % HBM roofline"
PREC = {"fp64": 0, "fp32": 1, "mixed": 2}


def solver_opts(a):
    """--solver-opts "key=value,...": extra Solver keyword arguments (ints)."""
    return {k: int(v) for k, v in (kv.split("=") for kv in a.solver_opts.split(",") if kv)}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="vflip", choices=["vflip", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--dt", type=float, default=0.01)
    ap.add_argument("--precision", default="fp32", choices=sorted(PREC))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-preconditioner arm")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched uneven-Poisson arm")
    ap.add_argument("--no-flip", action="store_true", help="skip the FLIP smoke arm")
    ap.add_argument("--no-nested", action="store_true", help="skip the nested-subdomain arm")
    ap.add_argument("--no-precisions", action="store_true", help="skip the fp64/mixed plain arms")
    ap.add_argument("--no-dropin", action="store_true", help="skip the host-CSR drop-in solve timing")
    ap.add_argument("--solver-opts", default="",
                    help="extra integer options of the headline Solver, e.g. coarse_tail=1,tile_sweep_max_cells=-1")
    ap.add_argument("--nested-ratio", type=int, default=4, choices=[2, 4],
                    help="refinement of the nested subdomain (4: a 256^3 subdomain over a 128^3 plume)")
    ap.add_argument("--learned-level", type=int, default=2)
    ap.add_argument("--learned-sweeps", type=int, default=2)
    ap.add_argument("--learned-capture", type=int, default=40)
    ap.add_argument("--learned-epochs", type=int, default=16)
    ap.add_argument("--cpu-budget", type=float, default=150.0, help="seconds for the reference arm's timed steps")
    ap.add_argument("--kernels", default=None,
                    help="instead of the step: per-kernel timings (comma list of advect, p2g, g2p, vcycle, unet, "
                         "hostlink, nested) at --n, "
                         "one JSON line each")
    ap.add_argument("--reps", type=int, default=5, help="timed repetitions per kernel (--kernels)")
    ap.add_argument("--unet-sizes", type=int, nargs="+", default=[32, 64, 128], help="network grids (--kernels unet)")
    ap.add_argument("--no-train", action="store_true", help="--kernels unet: forward only")
    return ap.parse_args()


def workload(a):
    return (f"smoke plume {a.n}^3 MAC grid, sphere obstacle r=0.15 + 5 solid walls, source sphere r=0.1 at "
            f"(0.5,0.1,0.5); step = RK2 trilinear advection of u,v,w,rho,T + sources/buoyancy + MGPCG "
            f"projection to 1e-6 (plain V(4,4) RBGS preconditioner)")


def config(a, n_gpus):
    out = {"workload": workload(a), "grid": a.n, "dt": a.dt, "precision": a.precision,
           "tolerance": 1e-6, "parallelism": f"replicas x{n_gpus}",
           "l2": "inputs larger than L2 (5 fields x 64 MB + solver vectors), no flush"}
    if a.solver_opts:
        out["solver_opts"] = a.solver_opts
    return out


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(n):
    """DRAM bytes per launch of the fine-level sweep from the ncu summary
    committed under profiles/, scaled to n^3 cells."""
    p = os.path.join(ROOT, "profiles", "rbgs_sweep_fp32_256.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_launch:"):
            b = float(line.split(":")[1].split()[0])
            return b * (n / 256.0) ** 3
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.path = os.path.join("/tmp", f"vflip_clocks_{os.getpid()}.csv")
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={gpu_id}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), parts[4:8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for _, _, r in rows for q in range(4) if r[q].lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


class Ranks:
    """One process per GPU: rank, world size and the two collectives the
    timing needs (a barrier, the max over ranks).  NCCL reduces a CUDA
    tensor, gloo (CPU tests) a CPU one; world size 1 needs no process group."""

    def __init__(self, backend="nccl", timeout_s=300):
        import datetime

        import torch.distributed as dist

        self.dist = dist
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        if self.world > 1:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max_over_ranks(self, x):
        if self.world == 1:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64, device="cuda" if self.backend == "nccl" else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


def replica_throughput(world, steps, ms_max):
    """Whole-job steps/s of `world` replicas that each ran `steps` steps, the
    slowest in `ms_max` milliseconds."""
    return world * steps / (ms_max * 1e-3)


def run_vflip(a):
    import numpy as np
    import torch

    from vflip_b200.plume import PlumeParams, PlumeSim
    from vflip_b200.solver import Solver

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ranks = Ranks("nccl")
    world, rank = ranks.world, ranks.rank
    barrier, max_over_ranks = ranks.barrier, ranks.max_over_ranks

    solver = Solver(precision=PREC[a.precision], device=local, **solver_opts(a))
    params = PlumeParams(n=a.n, dt=a.dt)
    sim = PlumeSim(solver, params)
    for _ in range(a.warmup):
        sim.step()
    torch.cuda.synchronize()

    props = torch.cuda.get_device_properties(local)
    clocks = ClockSampler(f"GPU-{props.uuid}" if getattr(props, "uuid", None) else str(local))
    time.sleep(0.3)
    iters, vcycles, resid = [], [], []
    launches0 = solver.launch_count
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        conv, st = sim.step()
        iters.append(st.iterations)
        vcycles.append(st.vcycles)
        resid.append(st.residual / max(st.rhs_norm, 1e-300))
    e1.record()
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    launches = solver.launch_count - launches0
    clk = clocks.stop()
    ms_max = max_over_ranks(ms)
    # the roofline's per-launch times: a separate pass of a few steps with the
    # library's events around every fine-level sweep (that pass runs the host
    # PCG loop, whose launches can carry events; the kernels are the same)
    solver.set_profiling(True)
    nprof = min(a.steps, 5)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record()
    for _ in range(nprof):
        sim.step()
    p1.record()
    torch.cuda.synchronize()
    # where a step's device time goes (per step, from the same events; spans
    # nest: the V-cycle holds the fine sweeps and the coarse part)
    breakdown = {"steps": nprof, "step_ms_with_events": p0.elapsed_time(p1) / nprof}
    for kind in ("vcycle", "coarse", "fine_sweep", "spmv", "update", "advect_field", "advect_pair"):
        cnt, kms = solver.profile_kernels(kind)
        breakdown[kind] = {"per_step": cnt / nprof, "ms_per_step": kms / nprof}
    n_sweeps, sweep_ms, cells = solver.profile_sweeps()
    solver.set_profiling(False)

    # end to end through the public API with host-resident state
    host = {k: torch.empty(sim.shapes[k], dtype=torch.float32, pin_memory=True) for k in sim.FIELDS}
    for k in sim.FIELDS:
        host[k].copy_(sim.f[k])
    sim.step_host(host)  # untimed: the first call sets up the copy streams
    sim.host_join()
    torch.cuda.synchronize()
    barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record()
    for _ in range(a.steps):
        sim.step_host(host)
    sim.host_join()  # the last step's downloads end inside the timed region
    e3.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e2.elapsed_time(e3))

    diag = solve_diagnostics(sim, local) if rank == 0 else None
    dropin = dropin_arm(sim, solver) if rank == 0 and world == 1 and not a.no_dropin else None
    out = None
    if rank == 0:
        peak, peak_kind = measured_peaks()
        avg_sweep_ms = sweep_ms / max(n_sweeps, 1)
        # the fine-level launches of one V(4,4) cycle: a zero-x sweep (no x read, 6 x 4 B per cell),
        # five plain sweeps and the fused z.r sweep (x_in, b, diag, xp, yp, zp read + x_out written,
        # 7 x 4 B) and the fused-prolongation sweep (+ the coarse x, 4 B per 8 cells), all FP32
        alg_bytes = (24 + 5 * 28 + 28 + 28.5) / 8 * cells
        achieved = alg_bytes / (avg_sweep_ms * 1e-3) / 1e9 if n_sweeps else None
        traffic = profile_traffic(a.n)
        out = {
            "metric": METRIC, "value": replica_throughput(world, a.steps, ms_max), "unit": "steps/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32" if a.precision != "fp64" else "fp64",
            "data": "synthetic (seeded plume scene, state evolved by the warm-up steps)",
            "config": config(a, world),
            "cells_steps_per_s": world * a.steps * a.n ** 3 / (ms_max * 1e-3),
            "solver": {"pcg_iterations_mean": float(np.mean(iters)), "vcycles_mean": float(np.mean(vcycles)),
                       "rel_residual_max": float(np.max(resid)), "levels": sim.last.levels, **diag},
            "roofline": {"bound": "hbm", "kernel": "rbgs_sweep_carry_kernel<float> (fine-level FP32 red-black sweep)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_sweep_ms,
                         "launches_timed": n_sweeps, "peak_kind": peak_kind},
            "e2e": {"value": replica_throughput(world, a.steps, e2e_ms), "unit": "steps/s",
                    "h2d_bytes_per_step": sim.host_bytes(), "d2h_bytes_per_step": sim.host_bytes()},
            "gpu_launches": launches,
            "clocks": clk,
            "step_breakdown": breakdown,
        }
        if dropin:
            out["dropin_host"] = dropin
        if not a.no_precisions and world == 1:
            out["precisions"] = precision_arm(a, sim, local, a.steps)
        if not a.no_cpu_baseline and world == 1:
            out["cpu_baseline"] = cpu_baseline(a, {k: sim.f[k].cpu().numpy().copy() for k in sim.FIELDS}, params)
        if not a.no_learned and world == 1:
            out["learned"] = learned_arm(a, sim, solver)
        if not a.no_batched and world == 1:
            out["batched"] = batched_arm(solver)
        if not a.no_flip and world == 1:
            out["flip"] = flip_arm(solver, a.steps)
            out["advection_forms"] = advection_arm(solver)
        if not a.no_nested and world == 1:
            out["nested"] = nested_arm(a.steps, device=local, ratio=a.nested_ratio)
    solver.close()
    ranks.close()
    return out


def learned_arm(a, sim, solver):
    """The learned arm on the same plume: the network corrects the previous
    pressure from its residual (VFLIP_LEARNED_RESID).  The next
    `learned_capture` projections run plain MGPCG and record training
    triples; the U-Net trains on the GPU (untimed); then `steps` steps each
    of three projections from the same states, interleaved step by step so
    that all three see the same flow: plain MGPCG from zero (the
    reference's solve), the warm start alone (the previous pressure scaled by
    the Ritz step, no network) and the learned warm start (previous pressure
    + the network's smoothed correction).  CUDA events around each step."""
    import numpy as np
    import torch

    from vflip_b200.learned import NO_NET, RESID, SOLVE, SWEEPS, LearnedPreconditioner

    lvl = a.learned_level
    pre = LearnedPreconditioner(solver, level=lvl, seed=0, sweeps=a.learned_sweeps, residual=True)
    for _ in range(a.learned_capture):
        sim.step(pre)
    torch.cuda.synchronize()
    t0 = time.time()
    losses = pre.train(epochs=a.learned_epochs, lr=1e-3)
    torch.cuda.synchronize()
    train_s = time.time() - t0
    modes = {"plain": None, "warm_start_only": SOLVE | RESID | NO_NET,
             "learned": SOLVE | RESID | SWEEPS(a.learned_sweeps)}
    res = {k: {"ms": [], "vc": [], "it": [], "net_ms": [], "fb": 0} for k in modes}
    for step in range(a.steps + 1):  # the first step is untimed: each arm's first call allocates its buffers
        sim.advect_and_force()
        u0 = {k: sim.f[k].clone() for k in ("u", "v", "w")}
        p0 = sim.pressure.clone()
        out = {}
        for name, mode in modes.items():
            for k in u0:
                sim.f[k].copy_(u0[k])
            sim.pressure.copy_(p0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            if mode is None:
                conv, _, st = sim.project()
            else:
                conv, _, st, ls = sim.project_learned(pre.net, mode, lvl)
                if step > 0:
                    res[name]["net_ms"].append(ls.net_ms)
                    res[name]["fb"] += int(ls.fallback)
            e1.record()
            torch.cuda.synchronize()
            if step > 0:
                res[name]["ms"].append(e0.elapsed_time(e1))
                res[name]["vc"].append(st.vcycles)
                res[name]["it"].append(st.iterations)
            out[name] = {k: sim.f[k].clone() for k in ("u", "v", "w")}, sim.pressure.clone()
        # the state continues from the learned projection
        for k in u0:
            sim.f[k].copy_(out["learned"][0][k])
        sim.pressure.copy_(out["learned"][1])
    # the rest of a step (advection, sources) is the same in every arm: the
    # plain step's time from the headline split into advection and projection
    summ = {k: {"projection_ms_mean": float(np.mean(v["ms"])), "vcycles_mean": float(np.mean(v["vc"])),
                "pcg_iterations_mean": float(np.mean(v["it"])),
                "network_ms_mean": float(np.mean(v["net_ms"])) if v["net_ms"] else 0.0, "fallbacks": v["fb"]}
            for k, v in res.items()}
    pl, ws, ln = summ["plain"], summ["warm_start_only"], summ["learned"]
    return {"arms": summ,
            "vcycle_ratio_learned_over_plain": ln["vcycles_mean"] / pl["vcycles_mean"],
            "projection_speedup_learned_over_plain": pl["projection_ms_mean"] / ln["projection_ms_mean"],
            "vcycle_ratio_learned_over_warm_start_only": ln["vcycles_mean"] / ws["vcycles_mean"],
            "projection_speedup_learned_over_warm_start_only": ws["projection_ms_mean"] / ln["projection_ms_mean"],
            "train_s": train_s, "train_final_loss": losses[-1], "train_first_loss": losses[0],
            "config": {"network_grid_level": lvl, "capture_steps": a.learned_capture, "epochs": a.learned_epochs,
                       "smoothing_sweeps": a.learned_sweeps,
                       "network": "4-level U-Net, 16/32/64/128 channels, BF16 tcgen05 convolutions",
                       "input": "residual of the previous pressure (level-L block averages) + fluid fraction",
                       "output": "correction of the previous pressure (Ritz-weighted with it)",
                       "steps": a.steps}}


def p2g_split(solver, sim, steps=2):
    """Device time per step of the P2G bucketing (histogram, scan, scatter,
    bucket sort, sorted copies) and of the gathers: CUDA events around them
    over `steps` further steps (with profiling on, the PCG loop runs from
    the host)."""
    solver.set_profiling(True)
    for _ in range(steps):
        sim.step()
    out = {k + "_ms": solver.profile_kernels(k)[1] / steps for k in ("p2g_sort", "p2g_gather")}
    solver.set_profiling(False)
    return out


def flip_arm(solver, steps, n=128, warmup=3):
    """The FLIP smoke scene at 128^3 (8 particles per cell jittered in the
    source sphere r = 0.12, sphere obstacle r = 0.15, FLIP/PIC 0.95, dt 0.01,
    MGPCG to 1e-6): advect_FLIP, P2G, projection, delta, G2P, reorder_FLIP
    per step, particles resident on the device; CUDA events around `steps`
    steps after `warmup` (reseeding fills every open cell to 8 particles)."""
    import torch

    from vflip_b200.flip import FlipParams, FlipSim

    sim = FlipSim(solver, FlipParams(n=n))
    for _ in range(warmup):
        sim.step()
    np0 = sim.num_particles
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    iters = []
    for _ in range(steps):
        conv, st = sim.step()
        iters.append(st.iterations)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out = {"grid": n, "steps_per_s": steps / (ms * 1e-3), "ms_per_step": ms / steps,
           "particles": sim.num_particles, "particles_at_start": np0,
           "particle_steps_per_s": sim.num_particles * steps / (ms * 1e-3),
           "pcg_iterations_mean": sum(iters) / len(iters)}
    out["p2g_per_step"] = p2g_split(solver, sim)
    del sim
    # the same scene with density/temperature on the 256^3 grid at h/2 (RK3
    # advection, gen_heat, buoyancy on the particles) inside every step
    sim = FlipSim(solver, FlipParams(n=n, smoke=True, alpha=0.1, beta=1.0))
    for _ in range(warmup):
        sim.step()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        sim.step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out["with_smoke_scalars"] = {"steps_per_s": steps / (ms * 1e-3), "ms_per_step": ms / steps,
                                 "scalar_grid": 2 * n, "particles": sim.num_particles}
    return out


def nested_arm(steps, device, n=128, warmup=3, ratio=4):
    """The nested-subdomain workload: a 128^3 FLIP plume (source sphere r =
    0.12 at (0.5, 0.1, 0.5), walls on five faces, open top, dt 0.005) with a
    subdomain over the central half at `ratio` x refinement (4: 256^3 cells at
    h/4, the refinement of the reference's own scene, main.cpp:63,71; 2:
    128^3 cells at h/2), coupled as SmokeSolver3D::time_step couples
    its SubDomainSolver: both particle passes, the main MGPCG to 1e-6 and the
    subdomain's to 1e-9, in the mixed-precision context (FP32 V-cycle with
    BF16 coarse operators, FP64 PCG scalars and coarsest solve).  CUDA events
    around `steps` steps after `warmup`.  Then one step from the reached state
    is repeated in an FP64 context: `fp64_rel_err` is max |v - v64| / max |v64|
    over the main and subdomain velocities."""
    import torch

    from vflip_b200.flip import NestedFlipSim, NestedParams
    from vflip_b200.solver import Solver

    prm = NestedParams(n=n, dt=0.005, obstacle_radius=0.0, ratio=ratio)
    with Solver(precision=PREC["mixed"], device=device) as s, Solver(precision=PREC["fp64"], device=device) as s64:
        sim = NestedFlipSim(s, prm)
        for _ in range(warmup):
            sim.step()
        np0, nsp0 = sim.num_particles, sim.num_sub_particles
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        it, sit = [], []
        for _ in range(steps):
            conv, st, sst = sim.step()
            it.append(st.iterations)
            sit.append(sst.iterations)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out = {"grid": n, "refinement": ratio, "subdomain_cells": list(sim.sdims), "subdomain_h": float(sim.sh),
               "steps_per_s": steps / (ms * 1e-3), "ms_per_step": ms / steps,
               "particles_main_pass": np0 + nsp0, "subdomain_particles": sim.num_sub_particles,
               "pcg_iterations_mean": sum(it) / len(it), "sub_pcg_iterations_mean": sum(sit) / len(sit),
               "precision": "mixed"}
        out["p2g_per_step"] = p2g_split(s, sim)
        # one step from this state in both precisions
        keep = {k: getattr(sim, k).clone() for k in ("particles", "sub_particles", "tracers")}
        keep_vel = [x.clone() for x in sim.vel] + [x.clone() for x in sim.sub_vel]
        keep_p = (sim.pressure.clone(), sim.sub_pressure.clone(), sim.steps)
        sim.step()
        mixed = [x.clone() for x in sim.vel] + [x.clone() for x in sim.sub_vel]
        for k, val in keep.items():
            setattr(sim, k, val)
        sim.vel, sim.sub_vel = keep_vel[:3], keep_vel[3:]
        sim.pressure.copy_(keep_p[0])
        sim.sub_pressure.copy_(keep_p[1])
        sim.steps = keep_p[2]
        sim.s = s64
        sim.sub_desc = s64.subdomain(sim.sdims, sim.sh, sim.bmin, *sim.sub_vel, sim.sphi)
        sim.step()
        ref = list(sim.vel) + list(sim.sub_vel)
        err = max(float((a - b).abs().max()) for a, b in zip(mixed, ref))
        scale = max(float(b.abs().max()) for b in ref)
        out["fp64_rel_err"] = err / scale if scale > 0 else None
        del sim
    return out


def advection_arm(solver, n=128, reps=20):
    """The grid advection forms and smoke scalars at the FLIP scene's size:
    SmokeSolver3D::advect (cubic-clamped u, v, w of a 128^3 MAC grid, one
    launch), advect_field (RK3) of density and temperature on their 256^3
    grid at h/2 (one shared backtrace), gen_heat on that grid and
    advect_tracers on 4 M tracers (RK3 + solid test, 32 B read + written per
    tracer), each timed
    with CUDA events on the library's stream (median of `reps` after 3
    warm-ups), in the solver's precision.  Algorithmic bytes: every output
    node reads its field value and writes one float (8 B), the velocity
    (read once) adds 4 B per face; the gathers behind each node (2 x 3
    trilinear velocity samples + 64 cubic nodes, or 3 x 3 + 2 trilinear
    samples) hit L1/L2, so these kernels are bound by load issue, not HBM."""
    import numpy as np
    import torch

    from vflip_b200 import scenes

    rng = np.random.default_rng(0)
    h = float(np.float32(1.0 / n))
    u, v, w = [torch.from_numpy(x).cuda() for x in scenes.random_velocity(n, n, n, rng, scale=1.0)]
    rho = torch.rand((2 * n,) * 3, device="cuda")
    temp = torch.rand_like(rho)
    r2, t2 = torch.empty_like(rho), torch.empty_like(rho)
    outs = tuple(torch.empty_like(x) for x in (u, v, w))

    def med(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    tracers = solver.emit_tracers(None, h, (1.0, 1.0, 1.0), (0.5, 0.5, 0.5), 0.3, 4_000_000, seed=0)
    phi = torch.full((n + 1,) * 3, 1.0, device="cuda")
    peak, _ = measured_peaks()
    faces = 3 * (n + 1) * n * n
    nodes2 = (2 * n) ** 3
    res = {}
    for name, fn, nodes, alg in (
            ("velocity_cubic_clamp", lambda: solver.advect_velocity_cubic_clamp(n, n, n, h, 0.01, u, v, w, outs=outs),
             faces, 8 * faces),
            ("rk3_density_temperature", lambda: solver.advect_rk3_linear(n, n, n, h, 0.01, u, v, w, rho, h / 2,
                                                                         field2=temp, out=r2, out2=t2),
             nodes2, 16 * nodes2 + 4 * faces),
            ("gen_heat", lambda: solver.gen_heat(rho, temp, h / 2, 0.01, 0.1, 0.1, (0.5, 0.1, 0.5), 0.12, 1.0, 1.0),
             nodes2, 16 * nodes2),
            ("advect_tracers", lambda: solver.advect_tracers(n, n, n, h, tracers, u, v, w, phi, 0.001, 0.1),
             tracers.shape[0], 32 * tracers.shape[0])):
        ms = med(fn)
        gbs = alg / (ms * 1e-3) / 1e9
        res[name] = {"ms": ms, "nodes": nodes, "gnodes_per_s": nodes / (ms * 1e-3) / 1e9, "alg_bytes": alg,
                     "achieved_gbs": gbs, "hbm_frac": gbs / peak if peak else None}
    res["grid"] = n
    return res


def batched_arm(solver, count=32, reps=2):
    """32 independent systems, sides uniform from {32..192}, random solid
    spheres, rhs = divergence of a smoothed Gaussian velocity (seeded), to
    1e-6, three ways: the whole batch as ONE persistent cooperative kernel
    (its work items autotuned on this batch first, untimed, and cached), as
    one CUDA graph of per-system device-side PCG loops, and one system after
    another; each timed from the first hierarchy build to the last result
    (CUDA events, best of `reps` after one untimed call)."""
    import numpy as np

    from vflip_b200 import scenes, tune
    from vflip_b200.solver import Solver

    systems, sides = scenes.batch_workload(solver, count=count, seed=0)
    best_cfg, table = tune.tune_batch(systems, sides, precision=solver.precision)
    res = {}
    pkw = {"batch_chunk": best_cfg["chunk"], "batch_ctas_per_sm": best_cfg["ctas_per_sm"]} if best_cfg else {}
    for name, mode, kw in (("persistent", 2, pkw), ("graph", 0, None), ("loop", 1, None)):
        s = Solver(precision=solver.precision, **kw) if kw is not None else solver
        best, stats, launch, ok = None, None, None, False
        for _ in range(reps + 1):  # the first call also creates the per-system contexts
            ok, _, st = s.batched_solve(systems, 1e-6, 100, mode=mode)
            ms = st[0].solve_ms
            if best is None or ms < best:
                best, launch = ms, s.last_ms
            stats = st
        if s is not solver:
            s.close()
        res[name] = (best, ok, stats, launch)
    cells = sum(x ** 3 for x in sides)
    p, g, l = res["persistent"], res["graph"], res["loop"]
    return {"systems": count, "sides": sides, "cells": cells, "persistent_ms": p[0], "persistent_kernel_ms": p[3],
            "graph_ms": g[0], "loop_ms": l[0], "graph_launch_ms": g[3],
            "speedup_persistent_over_graph": g[0] / p[0], "speedup_persistent_over_loop": l[0] / p[0],
            "speedup_graph_over_loop": l[0] / g[0], "all_converged": bool(p[1] and g[1] and l[1]),
            "iterations_mean": float(np.mean([x.iterations for x in g[2]])),
            "persistent_iterations_mean": float(np.mean([x.iterations for x in p[2]])),
            "iterations_equal_graph_loop": all(x.iterations == y.iterations for x, y in zip(g[2], l[2])),
            "cells_per_s_persistent": cells / (p[0] * 1e-3), "tuned": best_cfg, "tuning": table}


def csr_of_stencil(stencil):
    """Host CSR (rowstart, colindex, value) of a (4, nk, nj, ni) FP64
    stencil in the form SmokeSolver3D::pcg_projection hands to
    AMGPCGSolve: rows in cell order, columns sorted, the diagonal always
    present, off-diagonal couplings where non-zero (Smoke_solver3D.cpp
    :1040-1120, sparse_matrix.h:266-312)."""
    import numpy as np

    _, nk, nj, ni = stencil.shape
    n, sy, sz = ni * nj * nk, ni, ni * nj
    d, xp, yp, zp = (np.ascontiguousarray(stencil[c]).ravel() for c in range(4))
    r = np.arange(n, dtype=np.int64)
    i, j, k = r % ni, (r // ni) % nj, r // sz
    vals = np.zeros((n, 7))
    vals[sz:, 0] = zp[:-sz]
    vals[sy:, 1] = yp[:-sy]
    vals[1:, 2] = xp[:-1]
    vals[:, 3] = d
    vals[:, 4], vals[:, 5], vals[:, 6] = xp, yp, zp
    ok = np.stack([k > 0, j > 0, i > 0, np.ones(n, bool), i < ni - 1, j < nj - 1, k < nk - 1], axis=1)
    keep = ok & ((vals != 0) | (np.arange(7) == 3)[None, :])
    cols = r[:, None] + np.array([-sz, -sy, -1, 0, 1, sy, sz])[None, :]
    rowstart = np.zeros(n + 1, np.uint32)
    np.cumsum(keep.sum(axis=1), out=rowstart[1:])
    return rowstart, cols[keep].astype(np.uint32), vals[keep]


def dropin_arm(sim, solver, reps=3):
    """The reference-facing host-buffer call: the drop-in of
    ivock::AMGPCGSolve (vflip_amgpcg_solve_csr, AlgebraicMultigrid.h
    :189-197) on one plume step's pressure system as host CSR arrays, the
    call SmokeSolver3D::pcg_projection makes (Smoke_solver3D.cpp:1120).
    The call is synchronous (CSR pattern and symmetry checks and the
    conversion on host threads, one upload, the solve, the download), so it
    is timed by wall clock, median of `reps` after one untimed call, beside
    the same solve on device arrays (CUDA events)."""
    import numpy as np
    import torch

    state = {k: sim.f[k].clone() for k in sim.FIELDS}
    sim.advect_and_force()
    p, n = sim.p, sim.p.n
    stencil, rhs = solver.assemble(n, n, n, p.h, 0.0, sim.phi, sim.bdesc, sim.solid["u"], sim.solid["v"],
                                   sim.solid["w"], sim.f["u"], sim.f["v"], sim.f["w"])
    st_h, rhs_h = stencil.cpu().numpy(), rhs.cpu().numpy().ravel()
    rowstart, colindex, value = csr_of_stencil(st_h)
    solver.amgpcg_solve_csr(rowstart, colindex, value, rhs_h, p.tol, p.max_iterations, n, n, n)
    times = []
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ok, x_host, res, its = solver.amgpcg_solve_csr(rowstart, colindex, value, rhs_h, p.tol, p.max_iterations,
                                                       n, n, n)
        times.append((time.perf_counter() - t0) * 1e3)
    x_dev = torch.empty((n, n, n), dtype=torch.float64, device=rhs.device)
    solver.amgpcg_solve(stencil, rhs, p.tol, p.max_iterations, result=x_dev)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    solver.amgpcg_solve(stencil, rhs, p.tol, p.max_iterations, result=x_dev)
    e1.record()
    torch.cuda.synchronize()
    for k in sim.FIELDS:
        sim.f[k].copy_(state[k])
    ms = float(np.median(times))
    return {"call": "vflip_amgpcg_solve_csr (host CSR in, host result out)", "ms_per_solve": ms,
            "solves_per_s": 1e3 / ms, "device_ms_per_solve": e0.elapsed_time(e1), "converged": bool(ok),
            "iterations": its, "nnz": int(len(value)),
            "h2d_bytes": int(5 * 8 * n ** 3), "d2h_bytes": int(8 * n ** 3),
            "bitwise_equal_device_solve": bool(np.array_equal(x_host, x_dev.cpu().numpy().ravel())),
            "timing": f"wall clock around the synchronous call, median of {reps}"}


# the reference's own hierarchy (16^3 coarsest level, 200 red-black sweeps):
# in an FP64 context the V-cycle is the reference's bit for bit
REF_HIERARCHY = dict(coarse_sweeps=200, coarsest_max_unknowns=4096, coarsest_solver=1)


def solve_diagnostics(sim, device):
    """One more step, outside the timed region, whose projection is solved
    four ways on the same assembled system:
      * the benchmarked context (its precision and hierarchy);
      * an FP64 context with the reference's hierarchy to the same 1e-6: the
        reference's own answer (its V-cycle bit for bit, its iteration count);
      * an FP64 context to 1e-12: the converged solution;
      * an FP32 context with the reference's hierarchy, to 1e-6.
    The pressure errors split what FP32 arithmetic changes from what
    stopping at 1e-6 with another preconditioner changes: the reference's
    answer itself sits `ref_fp64_vs_converged` from the converged solution.
    Also both residual ratios and max |div u| before/after the projection."""
    import torch

    from vflip_b200.solver import Solver

    sim.advect_and_force()
    pre = {k: sim.f[k].clone() for k in ("u", "v", "w")}
    n, p = sim.p.n, sim.p
    before = float(sim.divergence(pre["u"], pre["v"], pre["w"]).abs().max())
    p32 = torch.zeros((n, n, n), dtype=torch.float64, device=sim.s.device)
    ok, _, st = sim.project(pressure=p32)
    after = float(sim.divergence(sim.f["u"], sim.f["v"], sim.f["w"]).abs().max())
    bench_u = [sim.f[k].clone() for k in ("u", "v", "w")]

    def solve(solver, tol, maxit=p.max_iterations):
        vel = [pre[k].clone() for k in ("u", "v", "w")]
        pr = torch.zeros_like(p32)
        ok_, _, st_ = solver.project(n, n, n, p.h, 0.0, sim.phi, sim.bdesc, sim.solid["u"], sim.solid["v"],
                                     sim.solid["w"], *vel, pressure=pr, tolerance_factor=tol, max_iterations=maxit)
        return pr, vel, st_

    with Solver(precision=0, device=device, **REF_HIERARCHY) as s64:
        p_ref, u_ref, st_ref = solve(s64, p.tol)
        p_conv, _, st_conv = solve(s64, 1e-12, 400)
    with Solver(precision=1, device=device, **REF_HIERARCHY) as s32r:
        p_r32, _, st_r32 = solve(s32r, p.tol)

    def rel(a, b):
        return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))

    vel_err = max(float((a - b).abs().max()) for a, b in zip(bench_u, u_ref)) / max(
        float(b.abs().max()) for b in u_ref)
    return {"rel_residual_inf": st.residual / st.rhs_norm, "iterations_last": st.iterations,
            "pressure_rel_l2_vs_reference_fp64_solve": rel(p32, p_ref),
            "pressure_rel_l2_vs_converged": rel(p32, p_conv),
            "ref_fp64_vs_converged": rel(p_ref, p_conv),
            "fp32_ref_hierarchy_vs_reference_fp64_solve": rel(p_r32, p_ref),
            "velocity_rel_max_vs_reference_fp64_solve": vel_err,
            "reference_iterations": st_ref.iterations, "fp32_ref_hierarchy_iterations": st_r32.iterations,
            "converged_iterations": st_conv.iterations,
            "max_abs_div_before": before, "max_abs_div_after": after}


def precision_arm(a, sim, device, steps):
    """The same plume, continued from the headline run's state, in the other
    precision modes of the plain MGPCG: steps/s (CUDA events, `steps` steps
    each after one untimed step), PCG iterations and V-cycles.  fp64 runs the
    reference's hierarchy (its bit-exact V-cycle): the like-for-like
    counterpart of the reference's FP64 solve."""
    import numpy as np
    import torch

    from vflip_b200.solver import Solver

    state = {k: sim.f[k].clone() for k in sim.FIELDS}
    out = {}
    for name, kw in (("fp64", dict(precision=0, **REF_HIERARCHY)), ("mixed", dict(precision=2)),
                     ("fp32", dict(precision=1))):
        if name == a.precision:
            continue
        with Solver(device=device, **kw) as s:
            old = sim.s
            sim.s = s
            for k in sim.FIELDS:
                sim.f[k].copy_(state[k])
            sim.step()
            its, vcs = [], []
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(steps):
                _, st = sim.step()
                its.append(st.iterations)
                vcs.append(st.vcycles)
            e1.record()
            torch.cuda.synchronize()
            sim.s = old
            ms = e0.elapsed_time(e1)
            out[name] = {"steps_per_s": steps / (ms * 1e-3), "ms_per_step": ms / steps,
                         "pcg_iterations_mean": float(np.mean(its)), "vcycles_mean": float(np.mean(vcs)),
                         "config": {k: v for k, v in kw.items()}}
    for k in sim.FIELDS:
        sim.f[k].copy_(state[k])
    return out


def _cpu_impl():
    import oracle

    r = oracle.reference()
    if r is not None:
        return r, "reference"
    return oracle.oracle(), "port"


def cpu_baseline(a, state, params):
    """One reference plume step on this state (bounded: a single step)."""
    import numpy as np

    from vflip_b200.plume import nodal_phi

    impl, kind = _cpu_impl()
    phi = nodal_phi(params)
    st = {k: np.ascontiguousarray(v) for k, v in state.items()}
    t0 = time.time()
    r = impl.smoke_step(a.n, params.h, params.dt, phi, st)
    wall = time.time() - t0
    secs = r[0] if kind == "reference" else wall
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())) if kind == "reference" else 1
    return {"value": 1.0 / secs, "unit": "steps/s", "cores": cores, "kind": kind,
            "sample": f"one full {a.n}^3 plume step from the GPU run's state (reference advect_field x5 + "
                      f"pcg_projection; {secs:.1f} s in reference code, {wall:.1f} s wall)"}


def run_reference(a):
    import numpy as np

    from vflip_b200 import scenes
    from vflip_b200.plume import PlumeParams, nodal_phi

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    impl, kind = _cpu_impl()
    params = PlumeParams(n=a.n, dt=a.dt)
    n = a.n
    su, sv, sw = scenes.face_shapes(n, n, n)
    st = {k: np.zeros(s, np.float32) for k, s in zip(("u", "v", "w", "rho", "temp"), (su, sv, sw, (n, n, n),
                                                                                     (n, n, n)))}
    phi = nodal_phi(params)

    def one():
        t0 = time.time()
        r = impl.smoke_step(n, params.h, params.dt, phi, st)
        wall = time.time() - t0
        return (r[0] if kind == "reference" else wall), wall

    warm = []
    for _ in range(max(1, min(a.warmup, 1))):  # one warm-up step: the reference is slow
        warm.append(one()[0])
    per = warm[-1]
    k = max(1, min(a.steps, int(a.cpu_budget // max(per, 1e-3))))
    times = [one()[0] for _ in range(k)]
    tot = sum(times)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())) if kind == "reference" else 1
    value = k / tot
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": a.gpus,
            "steps": k, "warmup": len(warm), "ms_per_step": 1e3 * tot / k, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp64+fp32 (reference: FP32 fields, FP64 solve)",
            "data": "synthetic (seeded plume scene)", "config": config(a, 1),
            "cpu_baseline": {"value": value, "unit": "steps/s", "cores": cores, "kind": kind,
                             "sample": f"{k} full {n}^3 plume steps from rest after {len(warm)} warm-up step(s) "
                                       f"(steps requested {a.steps}, bounded to ~{a.cpu_budget:.0f} s)"},
            "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def kernel_lines(a):
    """Per-kernel timings on seeded synthetic inputs (CUDA events on the
    library's stream after a warm-up call, L2 flushed between repetitions),
    each with its algorithmic bytes (or FLOPs) and the fraction of the
    measured peak:
      advect  the one-launch u, v, w advection (24 B/cell: u, v, w read once,
              written once) and the density/temperature pair (28 B/cell:
              u, v, w + both fields read, both written), n^3 cells, a smooth
              velocity field of peak |u| 0.4 (about 1 cell per step at dt 0.01);
      p2g     sort-by-cell P2G of 8 jittered particles per cell, all three
              components, sort included (24 B/particle + 24 B/cell);
      g2p     the FLIP update of the same particles (24 B/particle + 12 B/cell);
      unet    the U-Net forward (and a training step) on S^3 network grids
              (2 x 27 x c_in x c_out FLOP per voxel and layer)."""
    import numpy as np
    import torch

    from vflip_b200 import scenes
    from vflip_b200.solver import Solver

    n, dev = a.n, "cuda:0"
    peak, peak_kind = measured_peaks()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        tot = 0.0
        for r in range(a.reps):
            flush.fill_(r & 0xFF)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / a.reps

    def line(kernel, ms, alg, **kw):
        gbs = alg / (ms * 1e-3) / 1e9
        print(json.dumps({"kernel": kernel, "n": n, "ms": ms, "alg_bytes": alg, "achieved_gbs": gbs,
                          "hbm_frac": gbs / peak, "peak_gbs": peak, "peak_kind": peak_kind, **kw}), flush=True)

    what = a.kernels.split(",")
    h = np.float32(1.0 / n)
    rng = np.random.default_rng(0)
    T = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)  # noqa: E731
    with Solver(precision=PREC[a.precision], **solver_opts(a)) as s:
        if "advect" in what:
            vel = []
            for q, sh in enumerate(scenes.face_shapes(n, n, n)):
                k, j, i = np.meshgrid(*(np.arange(x, dtype=np.float32) for x in sh), indexing="ij")
                vel.append((0.4 * np.sin(0.05 * i + q) * np.cos(0.07 * j - q) * np.sin(0.03 * k + 2 * q)).astype(
                    np.float32))
            u, v, w = (T(x) for x in vel)
            outs = tuple(torch.empty_like(x) for x in (u, v, w))
            ms = timed(lambda: s.advect_velocity_rk2_linear(n, n, n, h, 0.01, u, v, w, outs=outs))
            gen = solver_opts(a).get("advect_kernel", 0) == 1
            line("advect_rk2_f_kernel x3 (u, v, w)" if gen else "advect_rk2_node_kernel (u, v, w, one launch)", ms,
                 24 * n ** 3)
            rho = T(rng.standard_normal((n, n, n)).astype(np.float32))
            tmp = T(rng.standard_normal((n, n, n)).astype(np.float32))
            o1, o2 = torch.empty_like(rho), torch.empty_like(tmp)
            ms = timed(lambda: s.advect_rk2_linear2(n, n, n, h, 0.01, u, v, w, rho, tmp, (0, 0, 0), out=o1, out2=o2))
            line(("advect_rk2_f_kernel" if gen else "advect_rk2_node_kernel") + " (density + temperature pair)", ms,
                 28 * n ** 3)
        if "p2g" in what or "g2p" in what:
            part = scenes.jittered_particles(n, n, n, h, 8, rng)
            part["vel"] = rng.standard_normal((len(part), 3)).astype(np.float32)
            npart = len(part)
            du, dv, dw = (T(x) for x in scenes.random_velocity(n, n, n, rng, scale=0.1))
            # two particle orders: shuffled (the worst case for the gathers)
            # and by cell (the order the FLIP step's reseeding leaves them in)
            cell = np.floor(part["pos"] / h + 0.5).astype(np.int64).clip(0, n - 1)
            by_cell = np.argsort(cell[:, 0] + n * (cell[:, 1] + n * cell[:, 2]), kind="stable")
            shuffled = rng.permutation(npart)
            for order, idx in (("shuffled", shuffled), ("cell order", by_cell)):
                parts = T(np.ascontiguousarray(part[idx]).view(np.uint8))
                if "p2g" in what:
                    ms = timed(lambda: s.particle_to_grid(n, n, n, h, parts))
                    # the split, from CUDA events around the bucketing and the
                    # gathers of one more call; the gathers' algorithmic bytes:
                    # the sorted positions and velocities read once (32 B per
                    # particle), six floats written per node index
                    s.set_profiling(True)
                    s.particle_to_grid(n, n, n, h, parts)
                    sort_ms = s.profile_kernels("p2g_sort")[1]
                    gather_ms = s.profile_kernels("p2g_gather")[1]
                    s.set_profiling(False)
                    gather_bytes = npart * 32 + 24 * (n + 1) ** 3
                    line(f"p2g (hash, sort, p2g3_kernel), particles in {order}", ms, npart * 24 + 24 * n ** 3,
                         particles=npart, sort_ms=sort_ms, gather_ms=gather_ms,
                         gather_hbm_frac=gather_bytes / (gather_ms * 1e-3) / 1e9 / peak)
                if "g2p" in what:
                    ms = timed(lambda: s.particle_from_grid(n, n, n, h, parts, du, dv, dw))
                    line(f"g2p_kernel, particles in {order}", ms, npart * 24 + 12 * n ** 3, particles=npart)
                del parts
        if "vcycle" in what:
            vcycle_lines(a, s, timed, line)
    if "unet" in what:
        unet_lines(a)
    if "hostlink" in what:
        hostlink_lines(a)
    if "nested" in what:
        nested_lines(a)


def nested_lines(a):
    """The nested arm's step (128^3 plume, 256^3 subdomain at 4x, mixed
    precision) alone: 3 warm-up steps, then --reps steps, each with its
    P2G split (CUDA events around the bucketing and the gathers)."""
    import torch

    from vflip_b200.flip import NestedFlipSim, NestedParams
    from vflip_b200.solver import Solver

    with Solver(precision=PREC["mixed"]) as s:
        sim = NestedFlipSim(s, NestedParams(n=128, dt=0.005, obstacle_radius=0.0, ratio=4))
        for _ in range(3):
            sim.step()
        for _ in range(a.reps):
            s.set_profiling(True)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            sim.step()
            e1.record()
            torch.cuda.synchronize()
            print(json.dumps({"kernel": "nested step (128^3 + 256^3 subdomain at 4x)", "ms": e0.elapsed_time(e1),
                              "p2g_sort_ms": s.profile_kernels("p2g_sort")[1],
                              "p2g_gather_ms": s.profile_kernels("p2g_gather")[1],
                              "particles_main_pass": sim.num_particles + sim.num_sub_particles}), flush=True)
            s.set_profiling(False)


def hostlink_lines(a):
    """The host link the end-to-end step crosses: one step's worth of fields
    (5 x n^3 FP32, pinned host memory) copied host to device, device to host,
    and both directions at once on two streams (CUDA events)."""
    import torch

    n = 5 * a.n ** 3
    h_in = torch.empty(n, dtype=torch.float32, pin_memory=True)
    h_out = torch.empty(n, dtype=torch.float32, pin_memory=True)
    d_in = torch.empty(n, dtype=torch.float32, device="cuda")
    d_out = torch.empty(n, dtype=torch.float32, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / a.reps

    def both():
        cur = torch.cuda.current_stream()
        s1.wait_stream(cur)
        s2.wait_stream(cur)
        with torch.cuda.stream(s1):
            d_in.copy_(h_in, non_blocking=True)
        with torch.cuda.stream(s2):
            h_out.copy_(d_out, non_blocking=True)
        cur.wait_stream(s1)
        cur.wait_stream(s2)

    gb = n * 4 / 1e9
    up = timed(lambda: d_in.copy_(h_in, non_blocking=True))
    down = timed(lambda: h_out.copy_(d_out, non_blocking=True))
    duplex = timed(both)
    print(json.dumps({"kernel": "host link (pinned, 5 fields)", "n": a.n, "bytes_each_way": n * 4,
                      "h2d_ms": up, "h2d_gbs": gb / up * 1e3, "d2h_ms": down, "d2h_gbs": gb / down * 1e3,
                      "both_ms": duplex, "both_gbs_each_way": gb / duplex * 1e3}), flush=True)


def vcycle_lines(a, s, timed, line):
    """One V(4,4)-cycle of the plume's own operator (the scene of the step,
    state evolved by a few steps), launched level by level from the host
    (vflip_vcycle), with the fine level's share: the V-cycle's device time,
    and its fine-level sweeps' algorithmic bytes over that time."""
    from vflip_b200.plume import PlumeParams, PlumeSim

    n = a.n
    sim = PlumeSim(s, PlumeParams(n=n, dt=a.dt))
    for _ in range(3):
        sim.step()
    sim.advect_and_force()
    p = sim.p
    st, rhs = s.assemble(n, n, n, p.h, 0.0, sim.phi, sim.bdesc, sim.solid["u"], sim.solid["v"], sim.solid["w"],
                         sim.f["u"], sim.f["v"], sim.f["w"])
    import torch

    s.vcycle(st, rhs)  # untimed: buffers and tensor maps
    s.set_profiling(True)
    for _ in range(a.reps):
        s.vcycle(st, rhs)
    torch.cuda.synchronize()
    cnt, ms = s.profile_kernels("vcycle")
    _, coarse_ms = s.profile_kernels("coarse")
    s.set_profiling(False)
    line("V(4,4)-cycle of the plume operator (all levels; CUDA events around the cycle, hierarchy build outside)",
         ms / max(cnt, 1), (24 + 6 * 28 + 28.5 + 24) * n ** 3, coarse_levels_ms=coarse_ms / max(cnt, 1),
         note="alg_bytes: the fine level's 8 sweeps and its restriction (FP32); the coarse levels add 1/7 of that")


UNET_LEVEL = {"E0A": 0, "E0B": 0, "E1A": 1, "E1B": 1, "E2A": 2, "E2B": 2, "B1": 3, "B2": 3, "D2A": 2, "D2B": 2,
              "D1A": 1, "D1B": 1, "D0A": 0, "D0B": 0, "OUT": 0}
UNET_LAYERS = [("E0A", 16, 16), ("E0B", 16, 16), ("E1A", 16, 32), ("E1B", 32, 32), ("E2A", 32, 64), ("E2B", 64, 64),
               ("B1", 64, 128), ("B2", 128, 128), ("D2A", 192, 64), ("D2B", 64, 64), ("D1A", 96, 32), ("D1B", 32, 32),
               ("D0A", 48, 16), ("D0B", 16, 16), ("OUT", 16, 16)]


def unet_forward_flops(S):
    """2 x 27 x c_in x c_out per voxel and layer (OUT counted at its 16 computed channels)."""
    return sum(2 * 27 * ci * co * (S >> UNET_LEVEL[nm]) ** 3 for nm, ci, co in UNET_LAYERS)


def measured_tflops():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def unet_lines(a):
    """U-Net forward (and training step) time on S^3 grids: 3 untimed
    forwards, then `reps` timed ones; also the program the convolution
    kernels' ncu profiles capture."""
    import torch

    from vflip_b200.learned import UNet

    peak = measured_tflops()
    net = UNet(seed=0)
    ev = lambda: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))  # noqa: E731
    for S in a.unet_sizes:
        g = torch.Generator(device="cuda").manual_seed(S)
        in2 = torch.randn((S, S, S, 2), device="cuda", generator=g)
        for _ in range(3):
            net.forward(in2)
        torch.cuda.synchronize()
        e0, e1 = ev()
        e0.record()
        for _ in range(a.reps):
            net.forward(in2)
        e1.record()
        torch.cuda.synchronize()
        fwd = e0.elapsed_time(e1) / a.reps
        tf = unet_forward_flops(S) / (fwd * 1e-3) / 1e12
        out = {"kernel": "unet forward (conv3_tc_kernel + pooling/upsampling)", "grid": S, "ms": fwd,
               "flops": unet_forward_flops(S), "achieved_tflops": tf, "tensor_frac": tf / peak[0],
               "peak_tflops": peak[0], "peak_kind": peak[1]}
        if not a.no_train:
            t2 = torch.randn((S, S, S, 2), device="cuda", generator=g)
            w = torch.ones((S, S, S), device="cuda")
            for _ in range(2):
                net.train_step(in2, t2, w, 1e-5, want_loss=False)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(a.reps):
                net.train_step(in2, t2, w, 1e-5, want_loss=False)
            e1.record()
            torch.cuda.synchronize()
            out["train_step_ms"] = e0.elapsed_time(e1) / a.reps
        print(json.dumps(out), flush=True)
    net.close()


def main():
    a = parse()
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    if a.kernels:
        kernel_lines(a)
        return
    out = run_reference(a) if a.impl == "reference" else run_vflip(a)
    if out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
