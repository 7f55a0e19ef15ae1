"""Liquid-step benchmark (one JSON line on rank 0).

Workload: the single world at scale — a 1024 x 1024 MAC grid with 200 WALL
disks (radii U[4, 24], centres uniform under the seed), WATER in the top half
at 4 particles per cell with Gaussian cell velocities (sigma 0.5 cells/step),
Earth's pull at dt 1/120 — stepped by the CUDA liquid step with the pressure
solved to a 1e-6 relative residual (||r||2/||b||2 of the CG residual, FP64
norms).

A step is one liquid step (encodeFluid's whole pass sequence).  `value` is
grid cells x steps / device time (CUDA events on the launch stream, the
world resident in HBM, 0.7 GB: larger than L2, so no flush is needed);
`e2e` is the same through the public API with every step's Params copied
host->device from pinned memory and the step's report read back, stepped
from the same saved state over the same trajectory.  A one-GPU run adds
`forms`: the batched workload (512 worlds of 64..512, every pass one launch
over all of them) and the served one (2000 resident worlds of 64..1024
under a 120 GB budget, Poisson requests, p50/p99 latency beside one world
a launch); --workload batched|served runs either alone.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--form fast|plain|persistent|mixed] [--workload single|batched|served]

With N > 1 (torchrun) every rank steps its own replica of the single world
(it does not shard: replicas only), or its cell-balanced share of N times
the batched or served worlds; timed as the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from worldinagrain_b200 import abi  # noqa: E402
from worldinagrain_b200 import world as W  # noqa: E402

METRIC = "Liquid-step Mcells/s at 1e-6 residual"
TOL = 1e-6
MAX_CYCLES = 64
FLAGS = abi.STEP_TOLERANCE | abi.STEP_F64_DOTS


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.lines = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if parts[3 + k].lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def make_world(args):
    if args.config == "disks":
        w = W.disks_world(1024, 1024, seed=args.seed)
    elif args.config == "dam":
        w = W.dam_break(256, 256, seed=args.seed)
    elif args.config == "column":
        w = W.obstacle_column(2048, 2048, seed=args.seed)
    else:
        raise SystemExit(f"unknown config {args.config}")
    return w


def params(world, step, seed):
    return W.make_params(world, frame=step, seed=seed, earth_g=world.config["earth_g"])


# Algorithmic bytes of one launch of each pass: the words the reference
# layout makes it read and write once (per active cell, fluid cell, face or
# particle), counted from the world after the step.  Active cells are the
# active blocks' 64 each.  The fast form's level kernels, per launch on a
# level of n cells.  A level cell holds four potential words of p bytes
# (px, py, rx, ry: FP32, 4; the mixed form's bf16, 2), five operator words
# of e bytes (rho, b0..b3: 4, or 2 in the mixed form's binary16) and,
# stored only in FP32, its diagonal (d = 4, mixed 0); level 0's restriction
# reads 40 B a cell in FP32 (the potentials, right-hand sides, density,
# coefficients and diagonal), 28 in the mixed form (its coefficients from
# their binary16 copies, no diagonal).  Down (restriction, then both colours of smoothing on
# chip): the four finer cells read, the coarse cell's px, py, rx, ry and
# rho written, 180 n in FP32; up (prolongation, then both colours): the
# level's words read, its way-up potentials written, the coarser level's
# density and way-up potentials read a quarter each, 51 n in FP32; the
# one-CTA coarse kernel on its first level: its potentials, right-hand
# sides and density read, its way-up potentials written, 28 n in FP32.
# Averaged over the launches of an iteration (s["levels"]: level_stats'
# cells of each level's launches; s["mixed"]: the mixed form).
def level_bytes(name, s):
    L = s.get("levels")
    if not L:
        return None
    p, e, d, c0 = (2, 2, 0, 28) if s.get("mixed") else (4, 4, 4, 40)
    cell = 4 * p + 5 * e + d
    down = [(4 * (c0 if i == 0 else cell) + 4 * p + e) * r for i, (r, _, _) in enumerate(L) if r]
    up = [(cell + 2 * p + (e + 2 * p) / 4) * m for _, m, _ in L if m]
    co = [(6 * p + e) * c for _, _, c in L if c]
    if name == "F_RESTRICT" and down:
        return int(sum(down)) // len(down)
    if name == "F_PROLONG" and up:
        return int(sum(up)) // len(up)
    if name == "F_COARSE" and co:
        return int(sum(co))
    return None


def level_stats(worlds, coarse_cells=4096):
    """Per level index l from 1: (cells a down launch takes, cells an up
    launch takes, cells the coarse kernel starts from), summed over the
    worlds, for the launch shape coarse_cells: a world's coarse kernel
    starts at its first level lc of at most that many cells (else its
    coarsest); its levels up to lc are restricted by the down kernel, those
    above lc also smoothed on the way up."""
    from collections import defaultdict
    res, smooth, coarse = defaultdict(int), defaultdict(int), defaultdict(int)
    for w in worlds:
        lv = w.L["levels"]
        lc = next((i + 1 for i, (a, b) in enumerate(lv) if a * b <= coarse_cells), len(lv))
        for i, (a, b) in enumerate(lv[:lc]):
            l = i + 1
            res[l] += a * b
            if l < lc:
                smooth[l] += a * b
            else:
                coarse[l] += a * b
    return [(res[l], smooth[l], coarse[l]) for l in sorted(res)]


# DRAM bytes (read + written) per algorithmic byte of a kernel, from one
# ncu capture each (dram__bytes_read.sum + dram__bytes_write.sum), keyed by
# (slot, mixed form). roofline.traffic is this ratio times a launch's
# algorithmic bytes: the capture's traffic scaled to the launch by the units
# it processes.
TRAFFIC_PER_ALG_BYTE = {
    # k_fDown on level 1 of the disks 1024x1024 world: 23.9 MB read, none
    # written; 262,144 cells x 180 B
    ("F_RESTRICT", False): (23.90272e6 / (262144 * 180), "k_fDown, level 1 (512x512) of the disks 1024x1024 world"),
    # k_fDown on levels 1-3 of one iteration of a 64-world batch, mixed form,
    # coarse cells 2048: 94.2 MB read and written; 153.3 MB algorithmic
    # (122 B a level-1 cell, 82 below: 1,043,904, 257,952 and 58,312 cells)
    ("F_RESTRICT", True): (94.191616e6 / 153.289936e6, "k_fDown, levels 1-3 of one iteration of a 64-world mixed batch"),
    # k_fRelax on the disks 1024x1024 world: 28.0 MB read, 0 written; 24.5 MB
    # algorithmic (the mixed form reads 12 B a cell less: its coefficients'
    # binary16 copies, no diagonal)
    ("F_RELAX", False): (28.0e6 / 24.5e6, "k_fRelax, the disks 1024x1024 world"),
    ("F_RELAX", True): (28.0e6 / 24.5e6, "k_fRelax, the disks 1024x1024 world"),
}


def traffic_of(name, alg, mixed=False):
    """(DRAM bytes a launch moves, where the figure comes from), or (None, None)."""
    t = TRAFFIC_PER_ALG_BYTE.get((name, bool(mixed)))
    if t is None or not alg:
        return None, None
    return int(round(t[0] * alg)), ("ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of " + t[1] +
                                    ", scaled to this launch's algorithmic bytes")


def algorithmic_bytes(name, s):
    A, Cf, N = s["active_cells"], s["fluid_cells"], s["particles"]
    lb = level_bytes(name, s)
    if lb is not None:
        return lb
    table = {
        # 10x10 tile of (field cell z, x; drift x; rim x2; share) in, pot out
        "RELAX": A * (16 + 4 + 8 + 4 + 4) + Cf * (8 + 8),
        "RELAX_SHIFTED": A * (16 + 4 + 8 + 4 + 4) + Cf * (8 + 8),
        # motion + state + affine read, the cell's and its faces' sums updated
        "GATHER": N * 48 + A * (2 * 4 * 4 + 3 * 4 * 2),
        "ADVECT": N * (32 + 16 + 16) + A * (2 * 16),
        "CG_APPLY": Cf * (16 + 4 + 4 + 4 + 4) + A * 4,
        "CG_UPDATE": Cf * (16 + 16 + 16),
        "CG_RHO": Cf * (16 + 4 + 4),
        "CG_DIRECTION": Cf * (8 + 8),
        "PROLONG_FINE": Cf * (16 + 8) + A * 8 // 4,
        "SCATTER": N * (48 + 48 + 8),
        "SYNC_PARTICLES": N * (48 + 48) + A * 16,
        "CLASSIFY": A * (16 + 32 + 32 + 12),
        "SET_FACES": A * 2 * (8 + 16 + 16 + 4),
        "PROJECT": A * 2 * (16 + 16 + 8),
        # the fast form's structure-of-arrays kernels (a float a cell per array)
        "F_RELAX": A * (4 + 8) + Cf * (32 + 8),
        # cgDirection with cgApply: z and the old p read, the new p and q written
        "F_APPLY_ALPHA": A * 12 + Cf * (8 + 4 + 16 + 8 + 1 + 4) + (A - Cf) * 8,
        "F_UPDATE": A * 4 + Cf * (16 + 4 + 24),
        "F_RHO_BETA": A * 4 + Cf * 12,
        "F_PROLONG_FINE": A * 4 + Cf * (8 + 16) + Cf // 4 * 12,
        "F_SETUP": A * (32 + 12 + 68),
    }
    return table.get(name)


def world_stats(world, coarse_cells=4096):
    blocks = world.blocks
    B = world.L["block_count"]
    active = int(blocks[4 * B + abi.COUNT_ACTIVE])
    rho = world.field_cells()[:, 0, 2]
    return {"active_cells": active * 64, "fluid_cells": int(np.sum(rho > 0)), "particles": int(world.sorted[0]),
            "levels": level_stats([world], coarse_cells)}


def cpu_baseline(world, args, budget_s):
    """The CPU oracle (a single-threaded port of the reference's passes) on
    the same world state, steps until about budget_s of work."""
    from oracle.oracle import Oracle
    w = world.copy()
    o = Oracle(w, W.element_table())
    steps, t0 = 0, time.perf_counter()
    while True:
        o.step(params(w, 10_000 + steps, args.seed), max_cycles=MAX_CYCLES, flags=FLAGS, tolerance=TOL)
        steps += 1
        if time.perf_counter() - t0 >= budget_s or steps >= args.cpu_steps_max:
            break
    dt = time.perf_counter() - t0
    return w.C * steps / dt / 1e6, steps, dt


def _reference_replica(args_d, worker, out_q):
    """One host core's replica of the reference arm: the oracle port stepping
    its own copy of the world, its warm-up, then timed steps until the
    budget or the step count is reached."""
    import argparse as ap_
    args = ap_.Namespace(**args_d)
    world = make_world(args)
    from oracle.oracle import Oracle
    o = Oracle(world, W.element_table())
    for s in range(1, args.warmup + 1):
        o.step(params(world, s, args.seed), max_cycles=MAX_CYCLES, flags=FLAGS, tolerance=TOL)
    steps, t0 = 0, time.perf_counter()
    while steps < args.steps:
        o.step(params(world, args.warmup + 1 + steps, args.seed), max_cycles=MAX_CYCLES, flags=FLAGS, tolerance=TOL)
        steps += 1
        if time.perf_counter() - t0 >= args.cpu_budget:
            break
    out_q.put((worker, world.C, steps, time.perf_counter() - t0))


def reference_cores(world_bytes):
    """Host cores the reference arm may use: one replica a core, as many as
    the cores and a third of the host's free memory allow (at most 64)."""
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    try:
        free = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
        cores = min(cores, max(1, int(free / 3 / max(world_bytes, 1))))
    except (ValueError, OSError, AttributeError):
        pass
    return max(1, min(cores, 64))


def run_reference(args, rank, world_size):
    """The reference arm: the oracle port (the reference's CPU restatement)
    timed on the host cores, one independent replica of the world a core
    (the oracle is sequential), the value the replicas' cells stepped per
    second of the slowest."""
    if rank != 0:
        return
    import multiprocessing as mp
    world = make_world(args)
    world_bytes = sum(getattr(world, n).nbytes for n in abi.BUFFER_NAMES)
    n = reference_cores(3 * world_bytes)
    t_w0 = time.perf_counter()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_reference_replica, args=(dict(vars(args)), k, q)) for k in range(n)]
    for p in procs:
        p.start()
    res = [q.get() for _ in procs]
    for p in procs:
        p.join()
    cells = sum(c * s for _, c, s, _ in res)
    dt = max(t for _, _, _, t in res)
    steps = min(s for _, _, s, _ in res)
    value = cells / dt / 1e6
    sample = (f"{n} replicas of the full {world.config['grid']} world, one a host core, each {args.warmup} warm-up "
              f"steps then timed steps up to {args.steps} or a {args.cpu_budget:.0f} s budget (fewest {steps}); "
              f"{time.perf_counter() - t_w0:.0f} s in all")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "Mcells/s", "n_gpus": world_size,
        "steps": steps, "warmup": args.warmup, "ms_per_step": round(dt / max(steps, 1) * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype_of(args.form),
        "data": "synthetic", "config": config_of(world, args),
        "cpu_baseline": {"value": round(value, 4), "unit": "Mcells/s", "cores": n, "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 4), "unit": "Mcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def gpu_index_of(torch, local_rank):
    gpu_index = torch.cuda.current_device()
    if "CUDA_VISIBLE_DEVICES" in os.environ and os.environ["CUDA_VISIBLE_DEVICES"].strip():
        try:
            gpu_index = int(os.environ["CUDA_VISIBLE_DEVICES"].split(",")[local_rank])
        except ValueError:
            pass
    return gpu_index


def run_batched(args, rank, world_size, local_rank, dist, torch, emit=True):
    """The batched multi-world workload: args.worlds independent worlds of
    uneven sizes (multi_worlds) resident together, every step one
    wig_batch_step of all of them (each pass one launch over all the
    worlds), solved to the same 1e-6 relative residual."""
    from worldinagrain_b200 import fluid, shard
    import ctypes as C
    # N ranks: N times the worlds, each rank its cell-balanced share (weak
    # scaling, no collective on the data path)
    n_all = args.worlds * world_size
    specs = W.multi_world_specs(n=n_all, seed=args.seed)
    all_cells = [s_[0] * s_[0] for s_ in specs]
    mine = shard.share_of(all_cells, rank, world_size)
    worlds = W.multi_worlds(n=n_all, seed=args.seed, only=mine)
    n = len(worlds)
    stream = torch.cuda.Stream()
    b = fluid.Batch(worlds, W.element_table())
    ids = (C.c_uint32 * n)(*range(n))
    P = (abi.Params * n)(*[params(w, 0, args.seed) for w in worlds])
    step_no = 0

    def step(extra=0):
        nonlocal step_no
        step_no += 1
        for k in range(n):
            P[k].frame = step_no
        b.step(ids, P, max_cycles=MAX_CYCLES, flags=FLAGS | extra, tolerance=TOL, stream=stream.cuda_stream)

    # the launch shapes tuned on the worlds' first steps, stepped by a batch
    # of their own (no result changes), so the timed trajectory is the one
    # the default shapes would step; then the warm-up
    tuned = None
    if not args.no_tune:
        from worldinagrain_b200 import tune
        tb = fluid.Batch(worlds, W.element_table())
        tune_no = 0

        def prof_step():
            nonlocal tune_no
            tune_no += 1
            for k in range(n):
                P[k].frame = tune_no
            return tb.step_profile(range(n), P, max_cycles=MAX_CYCLES, flags=FLAGS, tolerance=TOL,
                                   stream=stream.cuda_stream)

        shapes, trials = tune.autotune(tb, prof_step)
        tb.close()
        for name, v in shapes.items():
            b.set_launch(name, v)
        tuned = tuned_summary(shapes, trials)
    for name, v in args.launch.items():
        b.set_launch(name, v)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(gpu_index_of(torch, local_rank)) as clk:
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        barrier()
    ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = sum(all_cells) * args.steps / (ms / 1e3) / 1e6
    st = b.stats(range(n))
    launches_per_step = st[0].launches

    # end to end: every step's inputs in, every world's report out
    cycles, worst, worst_k = [], 0.0, -1
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
        sts = b.stats(range(n))
        cycles.append(max(x.cycles for x in sts))
        k = max(range(n), key=lambda i: sts[i].rel_residual)
        if sts[k].rel_residual > worst:
            worst, worst_k = sts[k].rel_residual, k
    e2e_s = time.perf_counter() - t0
    if worst > TOL:
        raise SystemExit(f"world {mine[worst_k]} (side {worlds[worst_k].W}) left {worst:.3e} > {TOL}")
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = sum(all_cells) * args.steps / e2e_s / 1e6
    h2d = 8 + ((4 * n + 7) // 8) * 8 + 136 * n
    d2h = 64 * n

    prof = {}
    for _ in range(args.profile_steps):
        step_no += 1
        for k in range(n):
            P[k].frame = step_no
        for key, (t_ms, cnt) in b.step_profile(range(n), list(P), max_cycles=MAX_CYCLES, flags=FLAGS, tolerance=TOL,
                                               stream=stream.cuda_stream).items():
            a0, c0 = prof.get(key, (0.0, 0))
            prof[key] = (a0 + t_ms, c0 + cnt)
    ws = {"active_cells": 0, "fluid_cells": 0, "particles": 0}
    for k, w in enumerate(worlds):
        b.download(k, names=("blocks", "field"))
        B = w.L["block_count"]
        ws["active_cells"] += int(w.blocks[4 * B + abi.COUNT_ACTIVE]) * 64
        ws["fluid_cells"] += int(np.sum(w.field_cells()[:, 0, 2] > 0))
    ws["particles"] = int(sum(x.particles for x in b.stats(range(n))))
    ws["levels"] = level_stats(worlds, b.get_launch("coarse_cells"))
    ws["mixed"] = args.form == "mixed"
    total = sum(v[0] for v in prof.values())
    ranked = sorted(prof.items(), key=lambda kv: -kv[1][0])
    top = next((k for k, _ in ranked if algorithmic_bytes(k, ws) is not None), ranked[0][0])
    t_ms, cnt = prof[top]
    per_launch_s = t_ms / cnt / 1e3
    alg = algorithmic_bytes(top, ws) or 0
    peak, peak_kind = peaks()
    achieved = alg / per_launch_s / 1e9 if per_launch_s > 0 else 0.0

    cpu = None
    if rank == 0 and not args.no_cpu:
        from oracle.oracle import Oracle
        done_cells, steps_done, t0 = 0, 0, time.perf_counter()
        for w in worlds:
            o = Oracle(w.copy(), W.element_table())
            o.step(params(w, 1, args.seed), max_cycles=MAX_CYCLES, flags=FLAGS, tolerance=TOL)
            done_cells += w.C
            steps_done += 1
            if time.perf_counter() - t0 >= args.cpu_budget:
                break
        dt = time.perf_counter() - t0
        cpu = {"value": round(done_cells / dt / 1e6, 4), "unit": "Mcells/s", "cores": 1, "kind": "port",
               "sample": f"the first step of {steps_done} of the {n} worlds on one host core, {dt:.1f} s"}
    b_shapes = b.launch_shapes()
    b.close()
    if rank == 0:
        sides = sorted(w.W for w in worlds)
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Mcells/s", "n_gpus": world_size,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype_of(args.form), "data": "synthetic",
            "config": {"workload": f"multi_worlds_{args.worlds}_per_gpu", "worlds": n_all, "cells": sum(all_cells),
                       "worlds_on_rank0": n, "sharding": "cell-balanced greedy partition, no data-path collective",
                       "sides": f"log-uniform {sides[0]}..{sides[-1]}, median {sides[n // 2]}", "seed": args.seed,
                       "liquid_per_cell": 4, "tolerance": TOL, "max_cycles": MAX_CYCLES,
                       "form": f"batched {args.form} form: one launch a pass over all worlds, CG loop in a graph WHILE node",
                       "launch": tuned["shapes"] if tuned else b_shapes,
                       "autotune": tuned,
                       "l2": "inputs larger than L2 (worlds resident in HBM, no flush)", "parallelism": "replicas"},
            "e2e": {"value": round(e2e, 3), "unit": "Mcells/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches_per_step * args.steps,
            "roofline": {"bound": "hbm", "kernel": top, "achieved": round(achieved, 1), "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic_of(top, alg, ws["mixed"])[0],
                         "traffic_source": traffic_of(top, alg, ws["mixed"])[1],
                         "algorithmic_bytes_per_launch": alg, "launch_ms": round(per_launch_s * 1e3, 5)},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "solve": {"cycles_max_mean": round(float(np.mean(cycles)), 2), "cycles_max": int(np.max(cycles)),
                      "rel_residual_worst": worst},
            "world": ws,
            "profile_ms_per_step": {k: round(v[0] / args.profile_steps, 4) for k, v in ranked[:12]},
            "profile_share": {k: round(v[0] / total, 4) for k, v in ranked[:12]},
        }
        if emit:
            print(json.dumps(line), flush=True)
        return line


def run_served(args, rank, world_size, local_rank, dist, torch, emit=True):
    """The served stream: args.worlds resident worlds (sides log-uniform
    64..1024), Poisson step requests at each rate of args.rates, admitted
    under a device-memory budget into two-lane continuously batched steps
    (lane pools lend each step its per-step memory); p50/p99 latency and
    Mcells/s per rate, beside the same stream served one world a launch."""
    from worldinagrain_b200 import serve, shard
    t0 = time.perf_counter()
    # N ranks: N times the worlds, each rank serving its cell-balanced share
    # and the requests for it (weak scaling; the ranks share only the
    # latencies, gathered on the host for the percentiles)
    n_all = args.worlds * world_size
    specs = W.multi_world_specs(n=n_all, lo=64, hi=1024, seed=args.seed)
    mine = shard.share_of([s_[0] * s_[0] for s_ in specs], rank, world_size)
    worlds = W.multi_worlds(n=n_all, lo=64, hi=1024, seed=args.seed, only=mine)
    t_build = time.perf_counter() - t0
    cells_of = [w.C for w in worlds]
    budget = int(args.budget_gb * 1e9)
    pool = int(args.pool_gb * 1e9)
    be = serve.GpuBackend(worlds, W.element_table(), FLAGS, MAX_CYCLES, TOL, pool_bytes=pool)
    srv = serve.Server(be, len(worlds), budget - 2 * pool)
    t0 = time.perf_counter()
    srv.preload()
    t_preload = time.perf_counter() - t0
    resident = len(srv.resident)
    # launch shapes tuned on profiled steps of the resident worlds (as many
    # as a lane's pool takes), then graphs captured and first steps seeded
    tuned = None
    if not args.no_tune:
        from worldinagrain_b200 import tune
        shapes, trials = be.autotune(list(srv.resident))
        tuned = tuned_summary(shapes, trials)
    srv.run(serve.poisson_arrivals(1000.0, 200, len(worlds), seed=99))
    rates = [float(r) for r in args.rates.split(",")]
    points = []
    with Clocks(gpu_index_of(torch, local_rank)) as clk:
        for rate in rates:
            n_req = int(min(max(rate * args.serve_seconds, 500), args.serve_max_requests))
            done = srv.run(serve.poisson_arrivals(rate, n_req, len(worlds), seed=args.seed + int(rate) + 7919 * rank))
            part = serve.latency_part(done, lambda k: cells_of[k])
            parts = [part]
            if dist:
                parts = [None] * world_size
                dist.all_gather_object(parts, part)
            pt = serve.merge_parts(parts)
            pt["rate"] = rate * world_size
            points.append(pt)
    # the one-world-at-a-time baseline (same kernels, one world a launch) at the lowest rate
    one = serve.Server(be, len(worlds), budget - 2 * pool, one_at_a_time=True)
    one.resident, one.resident_bytes = srv.resident, srv.resident_bytes
    rate0 = rates[0]
    arr = serve.poisson_arrivals(rate0, int(min(max(rate0 * args.serve_seconds, 300), 1500)), len(worlds),
                                 seed=args.seed + 7)
    part = serve.latency_part(one.run(arr), lambda k: cells_of[k])
    parts = [part]
    if dist:
        parts = [None] * world_size
        dist.all_gather_object(parts, part)
    base = serve.merge_parts(parts)
    base["rate"] = rate0 * world_size
    be.close()
    best = max(points, key=lambda p: p["mcells_per_s"])
    if rank == 0:
        line = {
            "metric": METRIC + "; served p50/p99 step latency", "value": best["mcells_per_s"], "unit": "Mcells/s",
            "n_gpus": world_size, "steps": sum(p["requests"] for p in points), "warmup": 200,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype_of(args.form),
            "data": "synthetic",
            "config": {"workload": f"served_{args.worlds}_worlds_per_gpu", "worlds": n_all,
                       "cells": sum(s_[0] * s_[0] for s_ in specs), "worlds_on_rank0": len(worlds),
                       "sides": "log-uniform 64..1024", "budget_gb": args.budget_gb, "lane_pool_gb": args.pool_gb,
                       "resident_worlds": resident, "resident_gb": round(srv.resident_bytes / 1e9, 2),
                       "build_s": round(t_build, 1), "preload_s": round(t_preload, 1), "tolerance": TOL,
                       "form": f"served {args.form} form: continuous batching over two lanes",
                       "autotune": tuned,
                       "arrivals": "Poisson, worlds uniform", "parallelism": "replicas"},
            "served": points,
            "one_at_a_time": base,
            "clocks": clk.summary(),
        }
        if emit:
            print(json.dumps(line), flush=True)
        return line


def tuned_summary(shapes, trials):
    """The autotuner's picks for the bench line; its per-candidate trial
    costs go to stderr as one JSON line (they would fill the line)."""
    print(json.dumps({"autotune_trials_ms_per_iteration": {
        k: [[v, None if c is None else round(c, 4)] for v, c in r] for k, r in trials.items()}}),
        file=sys.stderr, flush=True)
    from worldinagrain_b200 import tune
    return {"shapes": shapes, "steps": tune.steps_needed()}


def launch_overrides(items):
    """--launch KNOB=VALUE arguments as {knob: value}; SystemExit on an
    unknown knob or a value that is not a positive integer."""
    out = {}
    for it in items:
        name, _, v = it.partition("=")
        if name not in abi.LAUNCH_KNOBS or not v.isdigit() or int(v) <= 0:
            raise SystemExit(f"--launch {it}: want one of {', '.join(abi.LAUNCH_KNOBS)} = a positive integer")
        out[name] = int(v)
    return out


def dtype_of(form):
    """The arithmetic the form computes in: FP32 grids and vectors, FP64
    dots; the mixed form stores its coarse operator in binary16 and its
    levels' potentials in bf16."""
    return "bf16+f16+f32+f64" if form == "mixed" else "f32+f64"


def config_of(world, args):
    return {"workload": f"{world.config['workload']}_{world.config['grid']}", "grid": world.config["grid"],
            "seed": args.seed, "liquid_per_cell": world.L["liquid_per_cell"], "tolerance": TOL,
            "residual": "||r||2/||b||2 of the CG residual, FP64 norms", "max_cycles": MAX_CYCLES,
            "form": (f"{args.form} form over the reference's buffer layouts; FP32 vectors, FP64 dot products"),
            "l2": "inputs larger than L2 (world resident in HBM, no flush)", "parallelism": "replicas"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="disks")
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--profile-steps", type=int, default=2)
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--cpu-steps-max", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--form", default="fast", choices=["fast", "plain", "persistent", "mixed"])
    ap.add_argument("--workload", default="single", choices=["single", "batched", "served"])
    ap.add_argument("--worlds", type=int, default=None)
    ap.add_argument("--rates", default="1000,2000,5000,10000,20000,50000")
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--pool-gb", type=float, default=7.0)
    ap.add_argument("--serve-seconds", type=float, default=2.0)
    ap.add_argument("--serve-max-requests", type=int, default=4000)
    ap.add_argument("--no-tune", action="store_true", help="the default launch shapes, not the autotuner's")
    ap.add_argument("--no-forms", action="store_true",
                    help="the single world alone, without the batched and served summaries a one-GPU run adds")
    ap.add_argument("--launch", action="append", default=[], metavar="KNOB=VALUE",
                    help="a launch shape set on the measured handle after any tuning (coarse_cells, "
                         "level_per_sm, cg_per_sm, relax_per_sm); repeatable")
    args = ap.parse_args()
    args.launch = launch_overrides(args.launch)
    args.warmup = max(args.warmup, 3)
    global FLAGS
    if args.form == "plain":
        FLAGS = FLAGS | abi.STEP_PLAIN
    elif args.form == "persistent":
        FLAGS = FLAGS | abi.STEP_PERSISTENT
    elif args.form == "mixed":
        FLAGS = FLAGS | abi.STEP_MIXED

    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world_size)
        return

    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world_size > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local_rank))

    from worldinagrain_b200 import fluid

    if args.workload in ("batched", "served"):
        if args.worlds is None:
            args.worlds = 512 if args.workload == "batched" else 2000
        (run_batched if args.workload == "batched" else run_served)(args, rank, world_size, local_rank, dist, torch)
        if dist:
            dist.destroy_process_group()
        return

    world = make_world(args)
    stream = torch.cuda.Stream()
    g = fluid.LiquidStep(world, W.element_table(), stream=stream.cuda_stream)

    def flags_of(step):
        # the tiling parity fixed by the step's number, so a trajectory
        # replayed from a saved state repeats itself
        return FLAGS | abi.STEP_SHIFTED_SET | (abi.STEP_SHIFTED_FIRST if step % 2 else 0)

    step_no = 0
    # the fast forms' launch shapes tuned on the world's first steps, stepped
    # by a handle of their own (no result changes), so the timed trajectory
    # is the one the default shapes would step
    tuned = None
    if not args.no_tune and args.form in ("fast", "mixed"):
        from worldinagrain_b200 import tune
        tg = fluid.LiquidStep(world, W.element_table(), stream=stream.cuda_stream)
        tune_no = 0

        def prof_step():
            nonlocal tune_no
            tune_no += 1
            return tg.step_profile(params(world, tune_no, args.seed), max_cycles=MAX_CYCLES,
                                   flags=flags_of(tune_no), tolerance=TOL)

        shapes, trials = tune.autotune(tg, prof_step)
        tg.close()
        for name, v in shapes.items():
            g.set_launch(name, v)
        tuned = tuned_summary(shapes, trials)
    for name, v in args.launch.items():
        g.set_launch(name, v)
    for _ in range(args.warmup):
        step_no += 1
        g.step(params(world, step_no, args.seed), max_cycles=MAX_CYCLES, flags=flags_of(step_no), tolerance=TOL)
    g.stats()
    torch.cuda.synchronize()
    # the state after warm-up: the device-timed and the end-to-end runs both
    # step from it, over the same trajectory
    saved = g.download(world.copy())
    step_saved = step_no

    # ---- device-timed region: K steps, the world resident
    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(gpu_index_of(torch, local_rank)) as clk:
        barrier()
        with torch.cuda.stream(stream):
            e0.record(stream)
        for _ in range(args.steps):
            step_no += 1
            g.step(params(world, step_no, args.seed), max_cycles=MAX_CYCLES, flags=flags_of(step_no), tolerance=TOL)
        with torch.cuda.stream(stream):
            e1.record(stream)
        barrier()
    ms = e0.elapsed_time(e1)
    st = g.stats()
    launches_per_step = st.launches
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    cells = world.C
    value = cells * args.steps * world_size / (ms / 1e3) / 1e6

    # ---- end to end through the public API: params in, report out, every
    # step, from the same saved state
    g.upload(saved)
    step_no = step_saved
    cycles = []
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step_no += 1
        g.step(params(world, step_no, args.seed), max_cycles=MAX_CYCLES, flags=flags_of(step_no), tolerance=TOL)
        s2 = g.stats()
        cycles.append(s2.cycles)
        if s2.rel_residual > TOL:
            raise SystemExit(f"solve left {s2.rel_residual:.3e} > {TOL} after {s2.cycles} iterations")
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = cells * args.steps * world_size / e2e_s / 1e6

    # ---- per-pass device times of eagerly launched steps (events on the stream)
    prof = {}
    for _ in range(args.profile_steps):
        step_no += 1
        for k, (t_ms, n) in g.step_profile(params(world, step_no, args.seed), max_cycles=MAX_CYCLES, flags=FLAGS,
                                           tolerance=TOL).items():
            a, b = prof.get(k, (0.0, 0))
            prof[k] = (a + t_ms, b + n)
    g.download(world)
    ws = world_stats(world, g.get_launch("coarse_cells"))
    ws["mixed"] = args.form == "mixed"
    total = sum(v[0] for v in prof.values())
    ranked = sorted(prof.items(), key=lambda kv: -kv[1][0])
    top = next((k for k, _ in ranked if algorithmic_bytes(k, ws) is not None), ranked[0][0])
    t_ms, n = prof[top]
    per_launch_s = t_ms / n / 1e3
    alg = algorithmic_bytes(top, ws) or 0
    peak, peak_kind = peaks()
    achieved = alg / per_launch_s / 1e9 if per_launch_s > 0 else 0.0

    # ---- the plain drop-in (a kernel a reference pass) over the same steps
    # of the same trajectory, device-timed as above: the one-world baseline
    # the batched and served forms are compared with
    plain = None
    if world_size == 1 and not args.no_forms and args.form != "plain":
        def pflags(k):
            return flags_of(k) | abi.STEP_PLAIN
        g.upload(saved)
        g.step(params(world, step_saved + 1, args.seed), max_cycles=MAX_CYCLES, flags=pflags(step_saved + 1),
               tolerance=TOL)  # captures the plain form's graph
        g.stats()
        g.upload(saved)
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            p0.record(stream)
        for k in range(step_saved + 1, step_saved + 1 + args.steps):
            g.step(params(world, k, args.seed), max_cycles=MAX_CYCLES, flags=pflags(k), tolerance=TOL)
        with torch.cuda.stream(stream):
            p1.record(stream)
        torch.cuda.synchronize()
        pst = g.stats()
        pms = p0.elapsed_time(p1)
        plain = {"value": round(cells * args.steps / (pms / 1e3) / 1e6, 3), "unit": "Mcells/s",
                 "ms_per_step": round(pms / args.steps, 4), "steps": args.steps,
                 "form": "plain drop-in: a kernel a reference pass, in one CUDA graph a step",
                 "same_steps_as": "value (the same saved state and trajectory)",
                 "rel_residual_last": pst.rel_residual, "gpu_launches": pst.launches * args.steps}

    cpu = None
    if rank == 0 and not args.no_cpu:
        v, nsteps, dt = cpu_baseline(world, args, args.cpu_budget)
        cpu = {"value": round(v, 4), "unit": "Mcells/s", "cores": 1, "kind": "port",
               "sample": f"{nsteps} steps of the same {world.config['grid']} world state on one host core, {dt:.1f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Mcells/s", "n_gpus": world_size,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype_of(args.form), "data": "synthetic",
            "config": dict(config_of(world, args), launch=g.launch_shapes(), autotune=tuned),
            "e2e": {"value": round(e2e, 3), "unit": "Mcells/s", "h2d_bytes_per_step": 152, "d2h_bytes_per_step": 64},
            "gpu_launches": launches_per_step * args.steps,
            "roofline": {"bound": "hbm", "kernel": top, "achieved": round(achieved, 1), "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic_of(top, alg, ws["mixed"])[0],
                         "traffic_source": traffic_of(top, alg, ws["mixed"])[1],
                         "algorithmic_bytes_per_launch": alg, "launch_ms": round(per_launch_s * 1e3, 5)},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "solve": {"cycles_mean": round(float(np.mean(cycles)), 2), "cycles_max": int(np.max(cycles)),
                      "rel_residual_last": s2.rel_residual},
            "world": ws,
            "profile_ms_per_step": {k: round(v[0] / args.profile_steps, 4) for k, v in ranked[:12]},
            "profile_share": {k: round(v[0] / total, 4) for k, v in ranked[:12]},
        }
    g.close()
    if rank == 0 and world_size == 1 and not args.no_forms:
        line["forms"] = {"plain": plain} if plain else {}
        line["forms"].update(run_forms(args, rank, world_size, local_rank, dist, torch))
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_forms(args, rank, world_size, local_rank, dist, torch):
    """The one-GPU run's summaries of the batched and served forms, beside
    the single world: each its own workload (run_batched, run_served), in
    the mixed-precision form with tuned launch shapes, made smaller in steps
    and rates so the whole run stays within minutes."""
    import argparse as ap_
    global FLAGS
    out = {}
    b = ap_.Namespace(**vars(args))
    b.worlds, b.steps, b.warmup, b.no_cpu, b.profile_steps, b.form = 512, 10, 3, True, 1, "mixed"
    b.launch = {}  # the forms keep their own tuned shapes
    s = ap_.Namespace(**vars(args))
    s.worlds, s.rates, s.no_cpu, s.form = 2000, "1000,2000,20000", True, "mixed"
    saved = FLAGS
    FLAGS = abi.STEP_TOLERANCE | abi.STEP_F64_DOTS | abi.STEP_MIXED
    try:
        for name, fn, a in (("batched", run_batched, b), ("served", run_served, s)):
            try:
                ln = fn(a, rank, world_size, local_rank, dist, torch, emit=False)
                keep = ("value", "unit", "ms_per_step", "e2e", "config", "roofline", "solve", "served",
                        "one_at_a_time", "gpu_launches", "clocks")
                out[name] = {k: ln[k] for k in keep if k in ln}
            except Exception as e:  # a form that cannot run here is reported, not fatal
                out[name] = {"error": f"{type(e).__name__}: {e}"}
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
    finally:
        FLAGS = saved
    return out


if __name__ == "__main__":
    main()
