"""Benchmark: Mcell-steps/s of the full grid step on the 256^3 dam break.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--res 256]

Workload (one step = one full CGridFluidSolver::update): the 256^3 dam break
on the unit cube -- fluid in x < 0.4, y < 0.6, walls plus two static boxes of
side 0.2 on the floor, 8 particles per fluid cell (seeded), PIC/FLIP mix with
FLIP weight 0.95, CFL 1, linear transfers, RK3, gravity -9.8, dt = 1/60,
Jacobi-preconditioned CG to a relative residual of 1e-6 with at most 200
iterations, full velocity extrapolation.  The scene state (~3.5 GB) is far
larger than the 126 MB L2, so no L2 flush is needed between steps.

One process per GPU: with --gpus N > 1 and no torchrun environment the script
starts N ranks itself under torch.distributed.run.  For the dam break every
rank steps its own replica of the scene (weak scaling, no data-path
collective); for --workload serve|batch the scenes are placed on ranks by
their device-memory footprint.  The time is the maximum over ranks of the
CUDA-event time on each solver's stream.

--impl reference times the reference path on the host CPU (the reference has
no CPU implementation of the grid step, so its CPU restatement in oracle/ is
timed, FP64 with all host threads) on a bounded sample: one step of the same
dam-break layout at 128^3 per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "hybrid-fluid-simulation_b200")
sys.path.insert(0, PKG)

METRIC = "Mcell-steps/s at 256^3 (dam break, plain FP32 path)"
# dram__bytes_read.sum + dram__bytes_write.sum of kCgDirection and kCgUpdate,
# one launch each, ncu --set full on the 224^3 dam break (11.2 M cells) after 5
# steps.  The kernels stream only the fluid runs of the tile columns (the CG
# work list), so this is about a third of the 25 B/cell algorithmic figure,
# which counts every cell.
CG_DRAM_BYTES_PER_CELL = (42.556e6 + 0.884e6 + 50.508e6 + 0.303e6) / 224 ** 3
# Algorithmic bytes of one CFL substep per particle: position and v0 read and
# written (FP32 xyz each); the corner-table gathers hit L2.
SUBSTEP_BYTES_PER_PARTICLE = 48.0
# dram__bytes_read.sum + dram__bytes_write.sum of one kSubstep launch, ncu
# --set full on the 160^3 dam break (7.57 M particles), per particle
SUBSTEP_DRAM_BYTES_PER_PARTICLE = (243.88e6 + 133.72e6) / 7565040
UNIT = "Mcell-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--res", type=int, default=256)
    ap.add_argument("--precond", default="jacobi", choices=["jacobi", "identity", "mg"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-sample-res", type=int, default=128)
    ap.add_argument("--workload", default="dam-break", choices=["dam-break", "serve", "batch", "moving-boxes"],
                    help="dam-break: the 256^3 headline line; serve: Poisson stream of mixed-size requests "
                         "through the scene server vs each request run plain; batch: many uneven scenes at once")
    ap.add_argument("--mg-half", type=int, default=1, choices=[0, 1, 2],
                    help="multigrid storage: 0 FP32, 1 BF16 coarse levels, 2 BF16 level-0 smoothing iterates too")
    ap.add_argument("--mg-smooth", type=int, default=0, help="multigrid smoothing sweeps per level (0: library default)")
    ap.add_argument("--pressure-fp64", action="store_true",
                    help="accumulate the pressure in FP64 (divergence follows the CG residual)")
    ap.add_argument("--autotune", type=int, default=0, choices=[0, 1],
                    help="dam-break: 1 times the CG launch shapes at the first solve and keeps the fastest "
                         "(option autotune; done in the warm-up)")
    ap.add_argument("--sort-interval", type=int, default=0,
                    help="dam-break / moving-boxes: reorder the particles by cell every k steps (0: never)")
    ap.add_argument("--clamp-mode", type=int, default=None, choices=[0, 1],
                    help="boundary fix of the particles: 1 the first min(N, P) as the reference (default), 0 all")
    ap.add_argument("--ref-cpu", action="store_true",
                    help="reference arm: time the FP64 oracle port on the host cores even where the reference's "
                         "own CUDA build is present")
    ap.add_argument("--fp64-check", action="store_true",
                    help="moving-boxes: step the layout at 128x64x128 beside the FP64 oracle and report the per-step "
                         "error (and the oracle's time as the CPU baseline)")
    ap.add_argument("--requests", type=int, default=100, help="serve/batch: number of scenes")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: arrivals per second")
    ap.add_argument("--slots", type=int, default=16, help="serve/batch: concurrent scenes")
    ap.add_argument("--scene-steps", type=int, default=10, help="serve/batch: steps per scene")
    ap.add_argument("--no-plain", action="store_true", help="serve: skip the one-at-a-time comparison")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        cmd = ["nvidia-smi", f"--id={self.index}",
               "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
               "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
               "clocks_event_reasons.sw_power_cap",
               "--format=csv,noheader,nounits", "-lms", "200"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.rows.append(parts)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def rank_plan(n_gpus: int, port: int):
    """The command that runs this script on n_gpus ranks of this node (one
    process per GPU, rendezvous on 127.0.0.1)."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n_gpus}",
            "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]


def relaunch(n_gpus: int) -> int:
    """--gpus N > 1 outside torchrun: start the N ranks and wait for them."""
    import socket
    sk = socket.socket()
    sk.bind(("127.0.0.1", 0))
    port = sk.getsockname()[1]
    sk.close()
    return subprocess.run(rank_plan(n_gpus, port)).returncode


def init_ranks(world: int, local: int):
    """The process group of a multi-rank run (NCCL, short timeout), or None."""
    if world <= 1:
        return None
    import datetime
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return dist


def run_reference(args):
    """The reference arm, rank 0 only.  With the reference's own CUDA step
    built (oracle/_ref/refgpu) and a GPU visible, that step on the same
    workload as our arm; otherwise the oracle's FP64 restatement on the host
    cores, on a bounded sample."""
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refgpu
    if refgpu.available() and not args.ref_cpu:
        import torch
        if torch.cuda.is_available():
            run_reference_gpu(args)
            return
    import numpy as np
    import oracle
    import scenes

    n = args.cpu_sample_res
    threads = os.cpu_count() or 1
    oracle.lib().orc_set_num_threads(threads)
    sc = scenes.dam_break_256(n=n)
    o = oracle.Solver(sc.dt, sc.res, sc.origin, sc.spacing, dbl=1)
    for sdf, v in scenes.boundaries(sc):
        o.add_solid_boundary(sdf, v)
    dom = oracle.fluid_domain_from_bbox(sc.res, sc.origin, sc.spacing, *scenes.fluid_bbox(sc))
    o.set_fluid_domain_field(dom)
    o.set_advection(3, 2, 2, sc.cfl, sc.mixing, 1, 0)
    o.set_particles(oracle.seed_particles(sc.res, sc.origin, sc.spacing, dom, scenes.total_solid(sc), sc.per_cell,
                                          sc.seed))
    o.set_pcg(1, 1, 1e-6, 200)
    for _ in range(args.warmup):
        o.update()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.update()
    dt = time.perf_counter() - t0
    value = sc.n_cells * args.steps / dt / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"dam break, bounded CPU sample at {n}^3 (one step per timed step)",
                   "res": [n, n, n], "particles": o.num_particles, "pcg": "jacobi rel 1e-6 max 200"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} steps of the dam-break layout at {n}^3 (FP64 oracle)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_gpu(args):
    """The reference's CGridFluidSolver (its CUDA sources built unmodified
    for sm_100a) stepping the 256^3 dam break: walls and the two static boxes
    as SDF boundaries, the fluid domain from the bounding box, the PIC/FLIP
    mix seeded by the reference itself (8 per cell outside the solids, the
    count of our arm; linear transfers, CFL 1, mixing 0.05), its own pressure
    solve (identity preconditioner,
    sqrt(r.r) < 1e-3) with the iteration cap at the workload's 200.  Steps are
    timed with CUDA events on the default stream, where the reference
    launches everything."""
    import torch
    import refgpu
    import scenes
    torch.cuda.set_device(0)
    # the reference writes progress notes to stdout (e.g. EulerParticles.cpp:258);
    # they go to stderr here so that stdout carries the one JSON line
    sys.stdout.flush()
    saved_stdout = os.dup(1)
    os.dup2(2, 1)
    sc = scenes.dam_break_256(seed=0, n=args.res)
    t_setup = time.perf_counter()
    r = refgpu.RefSolver(sc.dt, sc.res, sc.origin, sc.spacing)
    for sdf, _ in scenes.boundaries(sc):
        r.add_solid_boundary(sdf)
    r.generate_fluid_domain_from_bbox(*scenes.fluid_bbox(sc))
    r.update_boundaries()
    n = r.set_mix_pic_flip(sc.per_cell, sc.cfl, sc.mixing)
    r.set_cg_iteration_cap(200)
    r.synchronize()
    setup_s = time.perf_counter() - t_setup
    for _ in range(args.warmup):
        r.update()
    r.synchronize()
    r.take_ax_calls()
    stream = torch.cuda.default_stream()
    clocks = ClockSampler(0)
    clocks.start()
    per_step, iters = [], []
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r.update()
        e1.record(stream)
        e1.synchronize()
        per_step.append(e0.elapsed_time(e1))
        iters.append(max(r.take_ax_calls() - 1, 0))
    clk = clocks.stop()
    ms = sum(per_step) / len(per_step)
    value = sc.n_cells / (ms / 1e3) / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded dam break)",
        "config": {"workload": f"dam break {args.res}^3, walls + two static boxes, 8 ppc, PIC/FLIP 0.95, "
                               "the reference's own pressure solve (identity-PCG, sqrt(r.r) < 1e-3) capped at 200",
                   "res": [args.res] * 3, "cells": sc.n_cells, "particles": n,
                   "implementation": "the reference's CGridFluidSolver, its CUDA sources built unmodified for "
                                     "sm_100a (oracle/refgpu/build.sh), driven through its C++ API",
                   "l2": "state > L2 (no flush needed)"},
        "cg_iterations_per_step": iters, "ms_per_step_each": per_step, "setup_s": setup_s, "clocks": clk,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": f"{args.steps} steps of the {args.res}^3 dam break after {args.warmup} warm-up "
                                   "steps: the reference's own CUDA step on this B200 (one host thread drives it)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    r.close()
    import ctypes
    ctypes.CDLL(None).fflush(None)
    os.dup2(saved_stdout, 1)
    os.close(saved_stdout)
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(n=64, steps=2):
    """Oracle FP64 on the host cores, bounded sample (same layout at n^3)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import scenes
    threads = os.cpu_count() or 1
    oracle.lib().orc_set_num_threads(threads)
    sc = scenes.dam_break_256(n=n)
    o = oracle.Solver(sc.dt, sc.res, sc.origin, sc.spacing, dbl=1)
    for sdf, v in scenes.boundaries(sc):
        o.add_solid_boundary(sdf, v)
    dom = oracle.fluid_domain_from_bbox(sc.res, sc.origin, sc.spacing, *scenes.fluid_bbox(sc))
    o.set_fluid_domain_field(dom)
    o.set_advection(3, 2, 2, sc.cfl, sc.mixing, 1, 0)
    o.set_particles(oracle.seed_particles(sc.res, sc.origin, sc.spacing, dom, scenes.total_solid(sc), sc.per_cell,
                                          sc.seed))
    o.set_pcg(1, 1, 1e-6, 200)
    o.update()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.update()
    dt = time.perf_counter() - t0
    return {"value": sc.n_cells * steps / dt / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} steps (after 1 warm-up) of the dam-break layout at {n}^3, FP64 oracle, {threads} threads"}


def serve_requests(args, rng, batch=False):
    """Request descriptions of the serving stream (C5) or the batch (C4)."""
    import numpy as np
    import hfgrid
    out = []
    for i in range(args.requests):
        if batch:
            # per-axis sizes U{32..128}, fluid fraction U(0.2, 0.5) as x < a, y < a with a = sqrt(frac)
            res = tuple(int(v) for v in rng.integers(32, 129, 3))
            a = float(np.sqrt(rng.uniform(0.2, 0.5)))
            fluid, spheres = (a, a, 1.0), []
        else:
            # cubic, side log-uniform in [32, 256]; 0-3 spheres in the free region
            n = int(round(float(np.exp(rng.uniform(np.log(32), np.log(256))))))
            res = (n, n, n)
            fluid = (0.4, 0.6, 1.0)
            spheres = []
            for _ in range(int(rng.integers(0, 4))):
                r = float(rng.uniform(0.05, 0.15))
                spheres.append((float(rng.uniform(0.45 + r, 0.95 - r)), float(rng.uniform(0.05 + r, 0.95 - r)),
                                float(rng.uniform(0.05 + r, 0.95 - r)), r))
        out.append(dict(res=res, spheres=spheres, fluid_max=fluid, seed=i))
    return out


def scene_descs(args, reqs, precond):
    import hfgrid
    return [hfgrid.scene_desc(r["res"], steps=args.scene_steps, spheres=r["spheres"], fluid_max=r["fluid_max"],
                              seed=r["seed"], precond=precond, tol_mode=hfgrid.TOL_RELATIVE, tol=1e-6,
                              max_iter=200) for r in reqs]


def run_batched(args, reqs, precond, device=0):
    """All scenes resident and stepped together through hfg_batch_*: the CFL
    substeps of every scene in one launch per substep, replayed from a graph."""
    import hfgrid
    descs = scene_descs(args, reqs, precond)
    t0 = time.perf_counter()
    b = hfgrid.Batch(descs, threads=args.slots, device=device)
    setup_s = time.perf_counter() - t0
    ms = b.step(args.scene_steps)
    cells = sum(int(r["res"][0]) * int(r["res"][1]) * int(r["res"][2]) for r in reqs)
    subs = [b.stats(i)["substeps"] for i in range(len(reqs))]
    b.close()
    step_s = sum(ms) / 1e3
    cs = float(cells * args.scene_steps)
    # like the server's wall time, from the first scene built to the last step
    wall_s = setup_s + step_s
    return {"scenes": len(reqs), "steps": args.scene_steps, "step_ms": ms, "cell_steps": cs, "setup_s": setup_s,
            "wall_s": wall_s, "mcell_steps_per_s": cs / max(wall_s, 1e-9) / 1e6,
            "mcell_steps_per_s_steps_only": cs / max(step_s, 1e-9) / 1e6,
            "substeps_max": max(subs) if subs else 0, "substeps_sum": sum(subs)}


def run_server(args, reqs, arrivals, slots, precond, device=0):
    """Submit `reqs` at their arrival times (seconds from start) to a server
    with `slots` concurrent scenes on `device`; returns its statistics."""
    import hfgrid
    srv = hfgrid.Server(slots=slots, budget_bytes=150 * 10**9, device=device)
    t0 = time.perf_counter()
    ids = []
    for r, at in zip(reqs, arrivals):
        dt = at - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        ids.append(srv.submit(scene_descs(args, [r], precond)[0]))
    srv.drain()
    st = srv.stats()
    infos = [srv.info(i) for i in ids]
    srv.close()
    st["mcell_steps_per_s"] = st["cell_steps"] / max(st["wall_s"], 1e-9) / 1e6
    st["failed_ids"] = [i for i, inf in zip(ids, infos) if inf["status"] != 2]
    return st


def run_serve(args):
    """C5 (serve) or C4 (batch) through the scene server, one JSON line.  With
    N ranks every rank builds the same request list, the scenes are placed on
    ranks by footprint (dist_util.assign_scenes, largest first under the
    150 GB budget of each GPU) and each rank serves its share on its own GPU;
    cell-steps add up and the wall time is the max over ranks."""
    import numpy as np
    import hfgrid
    import dist_util
    world, rank, local = dist_setup(args)
    pg = init_ranks(world, local)
    hfgrid.init(local)
    batch = args.workload == "batch"
    rng = np.random.default_rng(2024)
    reqs = serve_requests(args, rng, batch=batch)
    if batch:
        arrivals = [0.0] * len(reqs)
    else:
        arrivals = list(np.cumsum(rng.exponential(1.0 / args.rate, len(reqs))))
    budget = 150 * 10**9
    placed = list(range(len(reqs)))
    if world > 1:
        fp = [hfgrid.scene_bytes(r["res"], scene_particles(r), 1 + len(r["spheres"]), hfgrid.PRECOND_MG) for r in reqs]
        plan, rejected = dist_util.assign_scenes(fp, world, budget)
        placed = plan[rank]
        assert dist_util.agree([i for p in plan for i in p] + [-1] + rejected, device="cuda")
    mine = [reqs[i] for i in placed]
    at = [arrivals[i] for i in placed]
    clocks = ClockSampler(local)
    clocks.start()
    if pg is not None:
        pg.barrier()
    mixed = run_server(args, mine, at, args.slots, hfgrid.PRECOND_MG, local)
    batched = run_batched(args, mine, hfgrid.PRECOND_MG, local) if batch and mine else None
    clk = clocks.stop()
    plain = None
    if not args.no_plain:
        if pg is not None:
            pg.barrier()
        plain = run_server(args, mine, at, 1, hfgrid.PRECOND_JACOBI, local)
    if pg is not None:
        import torch.distributed as dist
        gathered = [None] * world
        dist.all_gather_object(gathered, {"mixed": mixed, "plain": plain, "clocks": clk, "n": len(mine),
                                          "batched": batched})
        pg.barrier()
        pg.destroy_process_group()
        if rank != 0:
            return
        mixed = merge_server_stats([g["mixed"] for g in gathered])
        plain = merge_server_stats([g["plain"] for g in gathered]) if plain is not None else None
        clk = gathered[0]["clocks"]
        parts = [g["batched"] for g in gathered if g["batched"]]
        if parts:
            wall = max(p["wall_s"] for p in parts)
            cs = sum(p["cell_steps"] for p in parts)
            batched = {"scenes": sum(p["scenes"] for p in parts), "cell_steps": cs, "wall_s": wall,
                       "mcell_steps_per_s": cs / max(wall, 1e-9) / 1e6, "ranks": len(parts)}
    line = {
        "metric": "Mcell-steps/s and step latency, " + ("batched uneven scenes" if batch else "served request stream"),
        "value": mixed["mcell_steps_per_s"], "unit": UNIT, "n_gpus": world, "higher_is_better": True,
        "scaling": "strong", "dtype": "f32 (MG preconditioner with BF16 coarse levels, FP64 dots)",
        "data": "synthetic (seeded)",
        "config": {"workload": ("C4 batch: %d scenes, axes U{32..128}, fluid fraction U(0.2,0.5), 8 ppc, %d steps"
                                % (len(reqs), args.scene_steps)) if batch else
                   ("C5 serve: %d requests, Poisson %.0f req/s, side log-uniform 32..256, 0-3 spheres, %d steps, "
                    "150 GB budget per GPU" % (len(reqs), args.rate, args.scene_steps)),
                   "slots": args.slots, "placement": "scenes by footprint over %d rank(s)" % world},
        "served": mixed, "clocks": clk,
    }
    if batched is not None:
        # all scenes resident, stepped together: one substep launch for all
        line["batched"] = batched
        line["batched_vs_streams"] = batched["mcell_steps_per_s"] / max(mixed["mcell_steps_per_s"], 1e-9)
    if plain is not None:
        line["plain"] = plain
        line["speedup_vs_plain"] = mixed["mcell_steps_per_s"] / max(plain["mcell_steps_per_s"], 1e-9)
    print(json.dumps(line), flush=True)


def scene_particles(r) -> int:
    """Particles of a served/batched request, bounded by 8 per cell of its
    fluid box (the server's own admission uses the same bound)."""
    fx, fy, fz = r["fluid_max"]
    nx, ny, nz = r["res"]
    return int(8 * int(fx * nx) * int(fy * ny) * int(fz * nz))


def merge_server_stats(parts):
    """Whole-job statistics of several ranks' servers: counts and cell-steps
    add up, the wall time is the longest, latency percentiles are the worst
    rank's (each rank holds its own step-time distribution)."""
    out = dict(parts[0])
    for k in ("submitted", "completed", "failed", "rejected", "cell_steps", "peak_bytes"):
        out[k] = sum(p[k] for p in parts)
    for k in ("wall_s", "step_ms_p50", "step_ms_p99", "request_ms_p50", "request_ms_p99"):
        out[k] = max(p[k] for p in parts)
    out["failed_ids"] = [i for p in parts for i in p["failed_ids"]]
    out["mcell_steps_per_s"] = out["cell_steps"] / max(out["wall_s"], 1e-9) / 1e6
    out["ranks"] = len(parts)
    return out


def run_moving_boxes(args):
    """C3: 512x256x512 dam break with three boxes on seeded sinusoidal paths,
    multigrid PCG (BF16 coarse levels, FP32 CG, FP64 dots), the box
    velocities set every step as in the viewer loop; per step the CG
    iterations and the divergence residual of the projection."""
    import torch
    import hfgrid
    import scenes
    hfgrid.init(0)
    res = (512, 256, 512)
    sc, paths = scenes.moving_boxes(res, seed=0)
    s = hfgrid.Solver(sc.dt, sc.res, sc.origin, sc.spacing)
    s.add_analytic_solid(hfgrid.SOLID_WALLS)
    for b in sc.solids:
        s.add_analytic_solid(hfgrid.SOLID_BOX, tuple(b.center) + tuple(b.size), b.velocity)
    mn, mx = scenes.fluid_bbox(sc)
    s.generate_fluid_domain_from_bbox(mn, mx)
    s.set_advection(hfgrid.ADV_MIX_PIC_FLIP, hfgrid.RK3, hfgrid.LINEAR, sc.cfl, sc.mixing)
    s.set_options(precond=hfgrid.PRECOND_MG, tol_mode=hfgrid.TOL_RELATIVE, tol=1e-6, max_iter=200,
                  advect_scalars=0, report_divergence=1, pressure_fp64=int(args.pressure_fp64),
                  sort_interval=args.sort_interval, mg_half=args.mg_half, clamp_mode=clamp_mode(args))
    s.seed_particles(sc.per_cell, sc.seed)
    stream = torch.cuda.ExternalStream(s.stream)
    t = 0.0
    per_step = []

    def step():
        nonlocal t
        for i, p in enumerate(paths):
            s.set_boundary_velocity(i + 1, p.velocity(t))
        s.update()
        t += sc.dt

    for _ in range(args.warmup):
        step()
    s.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    ms_total = 0.0
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        ms_total += ms
        st = s.stats()
        per_step.append({"ms": ms, "cg_iterations": st["cg_iterations"], "substeps": st["substeps"],
                         "rel_residual": st["cg_residual"] / max(st["cg_rhs_norm"], 1e-300),
                         "divergence_rel": st["divergence_l2"] / max(st["cg_rhs_norm"], 1e-300),
                         "divergence_max": st["divergence_max"]})
    clk = clocks.stop()
    N = sc.n_cells
    line = {"metric": "Mcell-steps/s, moving boxes 512x256x512 (multigrid PCG)",
            "value": N * args.steps / (ms_total / 1e3) / 1e6, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
            "dtype": "f32 (MG preconditioner with BF16 coarse levels, FP64 dots)", "data": "synthetic (seeded)",
            "config": {"workload": "C3: 512x256x512 dam break, three boxes (side 0.2) on sinusoidal paths "
                                   "(amplitude 0.1, period 2 s), 8 ppc, MG-PCG rel 1e-6 max 200",
                       "pressure": "fp64" if args.pressure_fp64 else "fp32",
                       "particle_sort_interval": args.sort_interval, "mg_half": args.mg_half,
                       "cells": N, "particles": s.num_particles},
            "per_step": per_step, "clocks": clk}
    del s
    if args.fp64_check:
        line["cpu_baseline"], line["fp64_check"] = moving_boxes_cpu_leg(args.pressure_fp64, args.mg_half)
    print(json.dumps(line), flush=True)


def moving_boxes_cpu_leg(pressure_fp64, mg_half=1, res=(128, 64, 128), steps=3):
    """The moving-boxes layout scaled down to 128x64x128, stepped on the GPU
    (the timed line's options) and in the FP64 oracle (Jacobi-PCG to 1e-10)
    side by side: the oracle's steps are the CPU baseline, and each step's
    GPU result is compared with them (velocity relative L2, marker agreement,
    largest particle-position difference)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import hfgrid
    import oracle
    import scenes
    threads = os.cpu_count() or 1
    oracle.lib().orc_set_num_threads(threads)
    sc, paths = scenes.moving_boxes(res, seed=0)
    g = scenes.gpu_solver(sc, precond=hfgrid.PRECOND_MG, tol_mode=hfgrid.TOL_RELATIVE, tol=1e-6, max_iter=200,
                          report_divergence=1, pressure_fp64=int(pressure_fp64), mg_half=mg_half)
    o = oracle.Solver(sc.dt, sc.res, sc.origin, sc.spacing, dbl=1)
    for sdf, v in scenes.boundaries(sc):
        o.add_solid_boundary(sdf, v)
    o.set_fluid_domain_field(oracle.fluid_domain_from_bbox(sc.res, sc.origin, sc.spacing, *scenes.fluid_bbox(sc)))
    o.set_advection(hfgrid.ADV_MIX_PIC_FLIP, 2, 2, sc.cfl, sc.mixing, 1, 0)
    pos, vel = g.particles()
    o.set_particles(pos, vel)
    o.set_pcg(1, 1, 1e-10, 20000)
    rows, cpu_s = [], 0.0
    for k in range(steps):
        t = k * sc.dt
        for i, p in enumerate(paths):
            g.set_boundary_velocity(i + 1, p.velocity(t))
            o.set_boundary_velocity(i + 1, p.velocity(t))
        g.update()
        t0 = time.perf_counter()
        o.update()
        cpu_s += time.perf_counter() - t0
        st = g.stats()
        vg, vo = g.velocity_field(), o.velocity_field()
        unknown = np.finfo(np.float32).max
        num = den = 0.0
        for a, b in zip(vg, vo):
            known = (a != unknown) & (b != unknown)  # faces both know
            num += float(np.sum((a[known].astype(np.float64) - b[known]) ** 2))
            den += float(np.sum(np.asarray(b[known], np.float64) ** 2))
        gp, _ = g.particles()
        op, _ = o.particles()
        rows.append({"step": k + 1, "vel_rel_l2": (num / max(den, 1e-300)) ** 0.5,
                     "markers_equal": float((g.markers() == o.markers()).mean()),
                     "max_pos_diff": float(np.abs(gp - op).max()), "cg_iterations": st["cg_iterations"],
                     "divergence_rel": st["divergence_l2"] / max(st["cg_rhs_norm"], 1e-300)})
    cells = sc.n_cells
    base = {"value": cells * steps / cpu_s / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} steps of the moving-boxes layout at {res[0]}x{res[1]}x{res[2]}, FP64 oracle, "
                      f"Jacobi-PCG to 1e-10, {threads} threads"}
    check = {"res": list(res), "oracle": "FP64, Jacobi-PCG rel 1e-10", "gpu": "the timed line's options",
             "per_step": rows}
    return base, check


def clamp_mode(args) -> int:
    return 1 if args.clamp_mode is None else args.clamp_mode


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch(args.gpus))
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "moving-boxes":
        run_moving_boxes(args)
        return
    if args.workload != "dam-break":
        run_serve(args)
        return
    run_dam_break(args)


def run_dam_break(args):
    """The headline line: the 256^3 dam break, one replica per rank."""
    import torch
    import hfgrid
    import scenes

    world, rank, local = dist_setup(args)
    pg = init_ranks(world, local)
    hfgrid.init(local)
    torch.cuda.set_device(local)
    precond = {"jacobi": hfgrid.PRECOND_JACOBI, "identity": hfgrid.PRECOND_IDENTITY, "mg": hfgrid.PRECOND_MG}[args.precond]
    sc = scenes.dam_break_256(seed=rank, n=args.res)
    opts = dict(precond=precond, tol_mode=hfgrid.TOL_RELATIVE, tol=1e-6, max_iter=200, advect_scalars=0,
                clamp_mode=clamp_mode(args), pressure_fp64=int(args.pressure_fp64),
                mg_smooth=args.mg_smooth, mg_half=args.mg_half,
                sort_interval=args.sort_interval, autotune=args.autotune)

    def warm_solver():
        """A solver in the state the timed steps start from: seeded, W steps in."""
        w = scenes.gpu_solver(sc, **opts)
        for _ in range(args.warmup):
            w.update()
        w.synchronize()
        return w

    s = warm_solver()
    stream = torch.cuda.ExternalStream(s.stream)

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    launches0 = s.launch_count
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        s.update()
    ev1.record(stream)
    ev1.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    launches = s.launch_count - launches0
    clk = clocks.stop()

    # one CG iteration (direction + update kernels) timed back-to-back on the
    # last system
    cg_ms = s.time_cg(40)

    # one more step, outside the timed region, with per-stage and per-kernel
    # device times and the convergence checks of the projection: the CG's
    # recurrence residual, ||b - A x|| recomputed in FP64, and the divergence
    # of the projected velocity
    s.set_options(**opts, report_divergence=1)
    s.enable_timing(True)
    s.update()
    st = s.stats()
    s.enable_timing(False)
    stage_ms = dict(zip(("boundaries", "advection", "forces", "markers", "rhs", "cg", "gradient", "extrapolation"),
                        (round(float(v), 3) for v in st["stage_ms"])))
    particle_ms = dict(zip(("g2p", "substeps", "p2g"), (round(float(v), 3) for v in st["particle_ms"])))
    bnorm = max(st["cg_rhs_norm"], 1e-300)
    conv = {"cg_iterations": st["cg_iterations"], "cg_converged": bool(st["cg_converged"]),
            "cg_rel_residual": st["cg_residual"] / bnorm, "cg_true_rel_residual_fp64": st["cg_true_residual"] / bnorm,
            "divergence_rel": st["divergence_l2"] / bnorm, "substeps": st["substeps"],
            "extrapolation_layers": st["extrapolation_layers"]}
    n = s.num_particles
    del s

    # e2e: the viewer loop of the reference (Application/main.cpp:74-93): the
    # frame's rigid-boundary motion in (3 floats per solid, from host values),
    # update(dt), then the particles (pos + vel) in pinned host buffers.  Each
    # pass runs on a fresh solver warmed up like the timed one, so it covers
    # the same simulation steps as `value`.
    e2e = None
    if not args.no_e2e:
        hpos = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
        hvel = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
        pos_np, vel_np = hpos.numpy(), hvel.numpy()
        nb = 1 + len(sc.solids)

        def e2e_pass(mirror):
            w = warm_solver()
            wstream = torch.cuda.ExternalStream(w.stream)
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            if mirror:
                w.set_particle_mirror(pos_np, vel_np)
            e0.record(wstream)
            for _ in range(args.steps):
                for i, sol in enumerate(sc.solids):
                    w.set_boundary_velocity(i + 1, sol.velocity)
                w.update()
                if not mirror:
                    w.copy_particles_into(pos_np, vel_np)
            e1.record(wstream)
            e1.synchronize()
            barrier()
            ms_ = e0.elapsed_time(e1)
            del w
            return ms_

        # through the particle mirror (each copy overlapped with the rest of the
        # step), and, for comparison, by a copy after each update
        e2e = {"ms": e2e_pass(True), "ms_copy_after": e2e_pass(False), "d2h": 24 * n, "h2d": 12 * (nb - 1)}

    def max_over_ranks(v):
        if pg is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    ms = max_over_ranks(ms)
    if e2e:
        e2e["ms"] = max_over_ranks(e2e["ms"])
        e2e["ms_copy_after"] = max_over_ranks(e2e["ms_copy_after"])
    cg_ms = max_over_ranks(cg_ms)
    sub_ms = max_over_ranks(float(st["particle_ms"][1]))

    if rank == 0:
        peaks = {}
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                peaks = json.load(f)
        except OSError:
            pass
        hbm = float(peaks.get("hbm_gbs", 6650.0))
        peak_source = "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks else "fallback 6650 GB/s"
        N = sc.n_cells
        value = N * args.steps * world / (ms / 1e3) / 1e6
        # the dominant kernel of the step: the CFL particle substep
        sub_launch_ms = sub_ms / max(conv["substeps"], 1)
        sub_bytes = SUBSTEP_BYTES_PER_PARTICLE * n
        sub_achieved = sub_bytes / (sub_launch_ms / 1e3) / 1e9
        # the CG pair, 25 B/cell per iteration (d, x, r read + markers + x, r, d written)
        algo_bytes = 25.0 * N
        achieved = algo_bytes / (cg_ms / 1e3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded dam break)",
            "config": {"workload": f"dam break {args.res}^3, walls + two static boxes, 8 ppc, PIC/FLIP 0.95, "
                                   f"{args.precond}-PCG rel 1e-6 max 200", "res": [args.res] * 3,
                       "cells": N, "particles": n, "l2": "state > L2 (no flush needed)",
                       "parallelism": f"replicas x{world}", "particle_sort_interval": args.sort_interval,
                       "cg_autotune": args.autotune, "clamp_mode": clamp_mode(args),
                       "mg_half": args.mg_half if args.precond == "mg" else None,
                       "convergence_one_more_step": conv,
                       "stage_ms_one_more_step": stage_ms, "particle_ms_one_more_step": particle_ms},
            "roofline": {"bound": "hbm", "kernel": "kSubstep (one CFL particle substep)",
                         "achieved": sub_achieved, "peak": hbm, "unit": "GB/s", "frac": sub_achieved / hbm,
                         "traffic": SUBSTEP_DRAM_BYTES_PER_PARTICLE * n,
                         "traffic_source": "ncu dram__bytes_read+write at 160^3, per particle, scaled",
                         "algorithmic_bytes_per_launch": sub_bytes,
                         "bytes_per_particle": SUBSTEP_BYTES_PER_PARTICLE, "ms_per_launch": sub_launch_ms,
                         "launches_per_step": conv["substeps"], "peak_source": peak_source,
                         "cg_pair": {"kernel": "kCgDirection + kCgUpdate (one CG iteration)", "achieved": achieved,
                                     "frac": achieved / hbm, "algorithmic_bytes_per_iter": algo_bytes,
                                     "ms_per_iter": cg_ms, "traffic": CG_DRAM_BYTES_PER_CELL * N,
                                     "traffic_source": "ncu dram__bytes_read+write at 224^3, per cell, scaled",
                                     "dram_frac": CG_DRAM_BYTES_PER_CELL * N / (cg_ms / 1e3) / 1e9 / hbm,
                                     "note": "the 25 B/cell figure counts every cell; the kernels stream only "
                                             "the fluid runs of the tile columns (the work list) and store at "
                                             "fluid cells only, so frac can pass 1 while dram_frac stays low"}},
            "clocks": clk,
            "gpu_launches": launches,
        }
        if e2e:
            line["e2e"] = {"value": N * args.steps * world / (e2e["ms"] / 1e3) / 1e6, "unit": UNIT,
                           "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"],
                           "what": "per step: solid velocities in, update() with the particle host mirror set "
                                   "(pos+vel to pinned host, the copy overlapped with the pressure solve)",
                           "value_copy_after_update":
                               N * args.steps * world / (e2e["ms_copy_after"] / 1e3) / 1e6}
        if world == 1 and args.cpu_sample_res > 0:
            try:
                line["cpu_baseline"] = cpu_baseline_sample(args.cpu_sample_res)
            except Exception as ex:  # the product number stands without it
                line["cpu_baseline"] = {"value": None, "error": str(ex)}
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
