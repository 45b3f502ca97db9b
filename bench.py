"""Benchmark of the coupled lattice update on B200: MLUPS of the fused
D3Q19-MRT + D3Q7 + pyrolysis step at 256^3 (FP32), one replica per GPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload pyro3d|pyro2d|flow2d] [--size S] [--precision fp32|fp16|fp64]

One JSON line on rank 0.  ``value`` is whole-job MLUPS (cells x steps x ranks /
max-over-ranks device time) with the state resident in HBM; ``e2e`` is the same
metric through the public API with a host->device copy of the boundary values
and a device->host read of the diagnostics every step.  Multi-GPU runs are
independent replicas (one seeded geometry per rank, no data-path collective):
weak scaling.  ``--impl reference`` times the CPU restatement of the reference
step (the Taichi reference cannot run here) with every host thread.
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
MIN_TIMED_MS = 2000.0   # device time the repeated timed blocks cover at least
MAX_REPEATS = 200       # bound on the repeats of the timed block
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pyro3d", choices=["pyro3d", "pyro2d", "flow2d", "sweep2d"])
    ap.add_argument("--instances", type=int, default=96, help="lattices of the sweep2d batch")
    ap.add_argument("--graph-steps", type=int, default=100,
                    help="steps per captured CUDA graph (even; 0: eager lbm_step calls)")
    ap.add_argument("--size", type=int, default=0, help="edge length override (default: the workload's)")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp16", "fp64"])
    ap.add_argument("--collision", default="")
    ap.add_argument("--e2e-steps", type=int, default=0, help="steps for the e2e leg (default: --steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--fp16-rounding", default="stochastic", choices=["stochastic", "nearest"],
                    help="FP16 storage: rounding of the temperature populations")
    ap.add_argument("--decomp", default="replicas", choices=["replicas", "slab"],
                    help="replicas: one lattice per GPU (weak scaling); slab: one lattice split along z "
                         "over the GPUs with a halo exchange every step (strong scaling)")
    ap.add_argument("--bulk", default="", choices=["", "tile", "list", "dense"],
                    help="bulk form of the lattice update (default: the library's choice)")
    return ap.parse_args(argv)


# ---------------------------------------------------------------- ranks (replicas, no data-path collective)
def rank_barrier(world: int) -> None:
    import torch.distributed as dist
    if world > 1:
        dist.barrier()


def max_over_ranks(v: float, world: int, device: str) -> float:
    """Largest per-rank value (the job's time is its slowest replica's)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_mlups(cells_per_rank: int, steps: int, world: int, ms_max: float) -> float:
    """Whole-job throughput: every rank updates its own lattice ``steps`` times."""
    return cells_per_rank * steps * world / (ms_max * 1e-3) / 1e6


def rank_seed(base: int, rank: int) -> int:
    """Each replica packs its own geometry."""
    return base + rank


def launches_per_step(cfg) -> int:
    """Kernels one lbm_step launches: bulk, boundary sides (if any), flip (pyrolysis)."""
    nbc = sum(1 for s in cfg.sides if s.active)
    return 1 + (1 if nbc else 0) + (1 if (cfg.thermal != "none" and cfg.pyro) else 0)


def make_workload(args, seed):
    from lbm_porouschem_b200 import workloads
    if args.workload == "sweep2d":        # the reference arm times one lattice of the sweep
        return workloads.sweep2d(1, seed0=seed, precision=args.precision)[0]
    if args.workload == "pyro3d":
        n = args.size or 256
        w = workloads.pyro3d(n, seed=seed, precision=args.precision, collision=args.collision or "mrt")
    elif args.workload == "pyro2d":
        nx = args.size or 512
        w = workloads.pyro2d(nx, nx // 2, seed=seed, precision=args.precision, collision=args.collision or "bgk")
    else:
        nx = args.size or 256
        w = workloads.flow2d(nx, nx // 2, seed=seed, precision=args.precision, collision=args.collision or "bgk")
    if args.bulk:
        w.cfg.bulk_form = args.bulk
    w.cfg.fp16_rounding = args.fp16_rounding
    return w


def describe(w, args):
    c = w.cfg
    lat = "D2Q9+D2Q5" if c.dim == 2 else "D3Q19+D3Q7"
    if c.thermal == "none":
        lat = "D2Q9" if c.dim == 2 else "D3Q19"
    return {
        "workload": f"{w.name} {lat} {c.collision.upper()}" + (" conjugate-heat+pyrolysis" if c.pyro else "")
                    + f" {c.precision}",
        "cells": c.ncells, "porosity": round(w.porosity, 4),
        "l2": "state larger than L2 (no flush needed)" if c.ncells * c.Q * 8 > 126e6 else "state fits in L2",
        **({"fp16_rounding": f"temperature populations {c.fp16_rounding}"} if c.precision == "fp16" else {}),
    }


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (read-only queries)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "", 1).isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "", 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------ CPU legs
def cpu_leg(w, steps_wanted, budget_s, warmup=1):
    """Time the CPU restatement (oracle/, FP32, OpenMP over all host threads) on the
    same workload; run as many of `steps_wanted` full steps as fit in budget_s."""
    from oracle import oracle
    oracle.build_oracle()
    o = oracle.Oracle(w.cfg, real="f32", threads=os.cpu_count())
    o.init(w.solid, w.reactive, **w.init)
    t0 = time.perf_counter()
    o.step(warmup)
    t_one = (time.perf_counter() - t0) / max(warmup, 1)
    n = max(1, min(steps_wanted, int(budget_s / max(t_one, 1e-9))))
    t0 = time.perf_counter()
    o.step(n)
    dt = time.perf_counter() - t0
    cores = o.threads()
    o.close()
    return w.cfg.ncells * n / dt / 1e6, n, cores, dt


def read_traffic(w):
    """Per-step DRAM traffic of the step kernels from the committed ncu summary, if any."""
    p = ROOT / "profiles" / f"traffic_{w.name}_{w.cfg.precision}.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_step:"):
            return float(line.split(":", 1)[1])
    return None


# ---------------------------------------------------------------- main
def main(argv=None):
    args = parse(argv)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        w = make_workload(args, args.seed)
        budget = 150.0
        mlups, n, cores, dt = cpu_leg(w, args.steps, budget, warmup=max(1, min(args.warmup, 2)))
        from lbm_porouschem_b200 import workloads as W
        line = {
            "impl": "reference", "metric": "coupled MLUPS", "value": round(mlups, 3), "unit": "MLUPS",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(dt / n * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded packing)",
            "config": describe(w, args),
            "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS", "cores": cores, "kind": "port",
                             "sample": f"{n} full steps of the same workload (C restatement of the "
                                       f"reference step, OpenMP; Taichi reference not runnable here)"},
            "e2e": {"value": round(mlups, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return 0

    if args.workload == "sweep2d":
        return sweep_main(args, world, rank, local)
    if args.decomp == "slab":
        return slab_main(args, world, rank, local)

    import torch
    import torch.distributed as dist
    from lbm_porouschem_b200 import workloads as W
    from lbm_porouschem_b200.lattice import Lattice

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=300))

    dev = f"cuda:{local}"

    def barrier():
        rank_barrier(world)

    w = make_workload(args, rank_seed(args.seed, rank))
    cfg = w.cfg
    stream = torch.cuda.Stream()
    lat = Lattice(cfg, device=f"cuda:{local}", stream=stream)
    lat.set_geometry(w.solid, w.reactive)
    lat.init(**w.init)
    bpl = W.bytes_per_lattice_update(cfg)
    alg_bytes = bpl * cfg.ncells                       # per step, every cell updated once
    sparse_bytes = W.algorithmic_bytes_per_step(cfg, w.solid)

    # ---- device-resident throughput (value): replays of a CUDA graph of graph_steps steps
    # when steps is a multiple of it (the launch gaps of small lattices disappear), else
    # one eager lbm_step call
    with torch.cuda.stream(stream):
        lat.step(args.warmup)
    use_graph = args.graph_steps > 0 and args.graph_steps % 2 == 0 and args.steps % args.graph_steps == 0
    if use_graph:
        lat.capture(args.graph_steps)
        lat.replay()                      # untimed: the captured steps run once
    stream.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)

    def timed_block() -> float:
        ev0.record(stream)
        if use_graph:
            for _ in range(args.steps // args.graph_steps):
                lat.replay()
        else:
            lat.step(args.steps)
        ev1.record(stream)
        ev1.synchronize()
        return ev0.elapsed_time(ev1)

    # the block of --steps steps is timed repeatedly until the blocks cover MIN_TIMED_MS of
    # device time (so the clock record has samples under load); the median block counts
    blocks = [timed_block()]
    while sum(blocks) < MIN_TIMED_MS and len(blocks) < MAX_REPEATS:
        blocks.append(timed_block())
    ms = float(np.median(blocks))
    clk = clocks.stop()
    barrier()
    torch.cuda.synchronize()
    ms_max = max_over_ranks(ms, world, dev)
    value = job_mlups(cfg.ncells, args.steps, world, ms_max)
    launches = args.steps * launches_per_step(cfg)

    # ---- end to end through the public API (host copies inside the timed region)
    k2 = args.e2e_steps or args.steps
    sides = cfg.sides
    pinned_diag = None
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    pending = None
    for _ in range(k2):
        lat.set_sides(sides)          # H2D: 6 side records from pinned host memory
        lat.step(1, diag=True)
        cur = lat.read_diag_async()   # D2H of this step's diagnostics, enqueued behind it
        if pending is not None:
            pinned_diag = pending.result()   # the previous step's values, while this step runs
        pending = cur
    pinned_diag = pending.result()
    e1.record(stream)
    e1.synchronize()
    wall = time.perf_counter() - t0
    ms_e2e = max(e0.elapsed_time(e1), wall * 1e3)
    ms_e2e = max_over_ranks(ms_e2e, world, dev)
    e2e_value = job_mlups(cfg.ncells, k2, world, ms_e2e)
    import ctypes
    from lbm_porouschem_b200 import _native as N
    h2d = 6 * ctypes.sizeof(N.lbm_side_desc)
    d2h = 10 * 8

    # ---- roofline of the step kernels (bulk + boundary): algorithmic bytes / event time
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    step_s = ms / args.steps * 1e-3
    achieved = alg_bytes / step_s / 1e9
    traffic = read_traffic(w)

    if rank == 0:
        line = {
            "metric": "coupled MLUPS", "value": round(value, 2), "unit": "MLUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
            "repeats": len(blocks), "timed_ms_total": round(sum(blocks), 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp32": "f32", "fp16": "f16-storage/f32", "fp64": "f64"}[cfg.precision],
            "data": "synthetic (seeded sphere/disk packing; one geometry per rank)",
            "config": {**describe(w, args), "bulk_form": lat.bulk_kernel, "parallelism": f"replicas x{world}",
                       "launch": f"CUDA graph of {args.graph_steps} steps" if use_graph else "lbm_step"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "algorithmic_bytes_per_step": alg_bytes, "bytes_per_lu": bpl,
                         "sparse_bytes_per_lu": round(sparse_bytes / cfg.ncells, 2),
                         "note": f"{bpl} B per lattice update (dense A/B pull count) x cells / device time of "
                                 f"the whole step (bulk + boundary + flip kernels); peak {peak_src}; "
                                 f"sparse_bytes_per_lu: lower bound when solid cells carry no flow "
                                 f"populations; traffic: DRAM bytes per step from ncu"},
            "e2e": {"value": round(e2e_value, 2), "unit": "MLUPS", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": k2},
            "gpu_launches": launches,
            "clocks": clk,
            "diag_last": {k: pinned_diag[k] for k in ("mass", "energy", "umax", "nonfinite")},
        }
        if world == 1 and not args.no_cpu_baseline:
            mlups, n, cores, dt = cpu_leg(w, 50, 20.0)
            line["cpu_baseline"] = {"value": round(mlups, 3), "unit": "MLUPS", "cores": cores, "kind": "port",
                                    "sample": f"{n} full steps of {w.name} (FP32 C restatement, OpenMP)"}
        print(json.dumps(line), flush=True)
    lat.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def sweep_main(args, world, rank, local):
    """Parameter sweep: ``--instances`` lattices of uneven sizes stepped as one batch,
    replayed from a CUDA graph of ``--graph-steps`` steps, against the same lattices
    launched one at a time."""
    import ctypes

    import torch
    import torch.distributed as dist
    from lbm_porouschem_b200 import _native as N
    from lbm_porouschem_b200 import workloads as W
    from lbm_porouschem_b200.lattice import Lattice, LatticeBatch

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=300))
    dev = f"cuda:{local}"
    ws = W.sweep2d(args.instances, seed0=rank_seed(args.seed, rank) * 1000, precision=args.precision,
                   collision=args.collision or "bgk")
    lats = []
    for w in ws:
        lat = Lattice(w.cfg, device=dev)
        lat.set_geometry(w.solid, w.reactive)
        lat.init(**w.init)
        lats.append(lat)
    torch.cuda.synchronize()
    cells = sum(w.cfg.ncells for w in ws)
    K = args.graph_steps + (args.graph_steps & 1)
    batch = LatticeBatch(lats)
    batch.step(max(4, args.warmup + (args.warmup & 1)))
    tuning = batch.tune(steps=4)           # persistent grid picked by timing (real steps)
    if batch.lattices[0].nsteps & 1:
        batch.step(1)
    batch.capture(K)
    batch.replay()                      # warm replay (brings the state level with the counters)
    batch.synchronize()
    reps = max(1, args.steps // K)
    rank_barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(batch.stream)
    for _ in range(reps):
        batch.replay()
    e1.record(batch.stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    ms_max = max_over_ranks(ms, world, dev)
    value = job_mlups(cells, reps * K, world, ms_max)

    # the same lattices launched one lattice at a time
    seq_steps = max(2, min(40, args.steps // 10))
    cur = torch.cuda.current_stream()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cur.wait_stream(batch.stream)
    s0.record(cur)
    for _ in range(seq_steps):
        for lat in lats:
            lat.step(1)
    s1.record(cur)
    s1.synchronize()
    seq_ms = max_over_ranks(s0.elapsed_time(s1), world, dev)
    seq_value = job_mlups(cells, seq_steps, world, seq_ms)
    batch.stream.wait_stream(cur)

    # end to end: per graph replay, the side records of every lattice go host -> device,
    # and every lattice's diagnostics come back
    reps2 = max(1, min(reps, 3))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    diag = None
    for _ in range(reps2):
        for lat in lats:
            lat.stream = batch.stream
            lat.set_sides(lat.cfg.sides)
        batch.replay()
        for lat in lats:
            lat.compute(diag=True)
            diag = lat.read_diag()
    wall_ms = (time.perf_counter() - t0) * 1e3
    for lat in lats:
        lat.stream = None
    e2e_ms = max_over_ranks(wall_ms, world, dev)
    e2e_value = job_mlups(cells, reps2 * K, world, e2e_ms)

    bytes_step = sum(W.bytes_per_lattice_update(w.cfg) * w.cfg.ncells for w in ws)
    pk = ROOT / "MEASURED_PEAKS.json"
    peaks = json.loads(pk.read_text()) if pk.exists() else {}
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = bytes_step / (ms / (reps * K) * 1e-3) / 1e9
    if rank == 0:
        sizes = {}
        for w in ws:
            sizes[f"{w.cfg.nx}x{w.cfg.ny}"] = sizes.get(f"{w.cfg.nx}x{w.cfg.ny}", 0) + 1
        line = {
            "metric": "coupled MLUPS", "value": round(value, 2), "unit": "MLUPS", "n_gpus": world,
            "steps": reps * K, "warmup": args.warmup, "ms_per_step": round(ms_max / (reps * K), 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp32": "f32", "fp16": "f16-storage/f32", "fp64": "f64"}[args.precision],
            "data": "synthetic (seeded disk packings, one parameter set per lattice)",
            "config": {"workload": f"sweep2d: {len(ws)} D2Q9+D2Q5 {ws[0].cfg.collision.upper()} "
                                   f"conjugate-heat+pyrolysis lattices, one batch, CUDA graph of {K} steps",
                       "cells": cells, "sizes": sizes, "parallelism": f"replicas x{world}",
                       "sequential_mlups": round(seq_value, 2), "sequential_steps": seq_steps,
                       "batch_vs_sequential": round(value / seq_value, 2),
                       "tuned_blocks_per_sm": batch.blocks_per_sm,
                       "tuning_ms_per_step": {str(k): round(v, 4) for k, v in tuning.items()},
                       "l2": "state larger than L2 (no flush needed)"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": None,
                         "note": "dense bytes per update x cells of all lattices / device time per batch step"},
            "e2e": {"value": round(e2e_value, 2), "unit": "MLUPS",
                    "h2d_bytes_per_step": len(ws) * ctypes.sizeof(N.lbm_side_desc),
                    "d2h_bytes_per_step": len(ws) * 10 * 8, "steps": reps2 * K,
                    "note": "one step = one graph replay of graph_steps lattice steps"},
            "gpu_launches": reps * K * (3 if ws[0].cfg.pyro else 2),
            "clocks": clk,
            "diag_last": {k: diag[k] for k in ("mass", "energy", "umax", "nonfinite")},
        }
        print(json.dumps(line), flush=True)
    batch.close()
    for lat in lats:
        lat.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def slab_main(args, world, rank, local):
    """One lattice split along z over the ranks (lbm_porouschem_b200.slab): each step is the
    tile-form update of every slab and its halo exchange (NCCL point-to-point between the
    ranks, device copies on one rank).  value = the lattice's cells x steps / max-over-ranks
    device time: strong scaling."""
    import torch
    import torch.distributed as dist
    from lbm_porouschem_b200.slab import SlabLattice, lattice_views
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=300))
    w = make_workload(args, args.seed)           # one geometry, the same on every rank
    cfg = w.cfg.replace(bulk_form="tile")
    sl = SlabLattice(cfg, device=f"cuda:{local}")
    sl.set_geometry(w.solid, w.reactive)
    sl.init(**w.init)
    stream = torch.cuda.current_stream()
    sl.step(args.warmup)
    rank_barrier(world)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    sl.step(args.steps)
    t1.record(stream)
    torch.cuda.synchronize()
    rank_barrier(world)
    ms = max_over_ranks(t0.elapsed_time(t1), world, f"cuda:{local}")
    views, _ = lattice_views(sl.lat)
    halo_bytes = sum(v[:, :sl.plan.halo].numel() * v.element_size() for v in views)
    if rank == 0:
        line = {
            "metric": "coupled MLUPS", "value": round(cfg.ncells * args.steps / (ms * 1e-3) / 1e6, 3),
            "unit": "MLUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": {"fp32": "f32", "fp16": "f16 storage, f32 arithmetic",
                                           "fp64": "f64"}[args.precision],
            "data": "synthetic (seeded packing)",
            "config": {**describe(w, args), "parallelism": f"slab z x{world}, halo {sl.plan.halo}",
                       "planes_per_rank": sl.plan.counts, "halo_bytes_per_neighbour_per_step": halo_bytes},
        }
        print(json.dumps(line), flush=True)
    sl.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
