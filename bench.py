#!/usr/bin/env python3
"""bench.py -- throughput of the MaHyCo hydro cycle on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload bisod3d|sedov3d|sod2d_lagrange]

A step is one compute-loop iteration (Lagrange step + ADI remap + CFL dt)
of one case.  Default workload: the plain 3D two-material BiSod, 256x64x64
cells on [0,1]x[0,0.25]^2, superbee limiter, FP64 (1 048 576 cells).  The
metric is cell-cycles/s = cells x timed iterations / device time.

Our arm: W untimed iterations, then K iterations enqueued on the case stream
and timed with CUDA events recorded on that stream (barrier + synchronize on
both sides, max over ranks).  The state (about 0.5 GB) is larger than L2, so
no flush is needed between iterations.  A second pass with events around
every kernel group gives the per-kernel roofline.  `e2e` runs the same K
iterations through the public C ABI from host parameters to host results:
case creation and device init, one status read-back per iteration (time,
deltat, flags) and the download of the final cell and node fields.

Reference arm (--impl reference): the reference cannot be built here (it
needs the Arcane framework), so the arm times the CPU oracle, a sequential
restatement of the reference algorithm, on a bounded slab of the same
workload; under torchrun only rank 0 runs it.

N > 1: one process per GPU, each advancing its own replica of the case
(weak scaling, no data-path collective); value = all ranks' cell-cycles /
max-over-ranks time.
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
sys.path.insert(0, ROOT)

METRIC = "cell-cycles/s and p50/p99 solve latency, batched/served vs plain, 1 B200"

WORKLOADS = {
    # name: (builder kwargs, description)
    "bisod3d": ("plain 3D BiSod 256x64x64, 2 materials, ADI remap, superbee, FP64", 2),
    "sedov3d": ("plain 3D Sedov 384^3, 1 material, ADI remap, minmod, FP64", 1),
    "sod2d_lagrange": ("plain 2D Lagrange Sod 200x10, FP64", 1),
}


def build_params(name: str, scale: float = 1.0):
    from mahyco_b200.cases import sod, sedov, SUPERBEE, MINMOD
    if name == "bisod3d":
        ny = max(1, int(round(64 * scale)))
        return sod(dim=3, n=(256, ny, ny), L=(1.0, 0.25 * ny / 64, 0.25 * ny / 64), bi=True,
                   limiter=SUPERBEE, deltat_init=1e-5)
    if name == "sedov3d":
        n = max(2, int(round(384 * scale)))
        p = sedov(dim=3, n=(n, n, n), L=1.2 * n / 384, limiter=MINMOD, energy=0.2468, p0=1e-6)
        return p
    if name == "sod2d_lagrange":
        return sod(dim=2, n=(200, 10), L=(1.0, 0.05), bi=False, remap=False, deltat_max=1e-4)
    raise ValueError(name)


# algorithmic bytes per launch of each kernel group (compulsory traffic of
# the live fields, FP64): see DESIGN.md "Roofline model"
def stage_bytes(stage: str, dim: int, ne: int, ncell: int, nnode: int) -> float:
    nv = 3 * ne + 1
    per = {
        "lagrange_nodes": 13 * nnode + 2 * ncell,
        "lagrange_cells": (6 + nv + 2) * ncell + 3 * nnode,
        "sweep_cells": (2 * nv + ne) * ncell + (dim + 1) * nnode,
        "sweep_nodes": 11 * nnode + ne * ncell,
        "finalize_cells": (nv + 1 + 7) * ncell,
        "finalize_nodes": 8 * nnode + ncell,
        "delta_t": 3 * nnode + 2 * ncell,
    }[stage]
    return 8.0 * per


def launches_per_cycle(p) -> int:
    dirs = sum(1 for n in ((p.nx, p.ny, p.nz) if p.dim == 3 else (p.nx, p.ny)) if n > 1)
    if p.with_projection:
        return 2 + 2 * dirs + 2 + 2
    return 2 + 2


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 8:
                self.samples.append(f)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[4 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def peaks() -> dict:
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        return {"hbm_gbs": 6650.0, "source": "fallback"}


def profile_traffic(workload: str) -> dict:
    """Per-launch DRAM traffic of the kernels measured by ncu (profiles/)."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "traffic.json"))).get(workload, {})
    except OSError:
        return {}


def cpu_baseline(workload: str, cycles: int = 20) -> dict:
    """The CPU oracle on a bounded slab of the workload (same per-cell work),
    about 10 s of single-core work."""
    from tests.oracle import Oracle
    scale = {"bisod3d": 0.5, "sedov3d": 0.125, "sod2d_lagrange": 1.0}[workload]
    if workload == "sod2d_lagrange":
        cycles = 2000
    p = build_params(workload, scale)
    o = Oracle(p, cr_pow=False)
    o.init()
    o.iterate(1)
    t0 = time.perf_counter()
    o.iterate(cycles)
    dt = time.perf_counter() - t0
    return {"value": p.ncell * cycles / dt, "unit": "cell-cycles/s", "cores": 1, "kind": "port",
            "sample": f"{cycles} iterations of a {p.nx}x{p.ny}x{p.nz if p.dim == 3 else 1} slab of the same "
                      f"workload ({p.ncell} cells), single-threaded sequential oracle"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    base = cpu_baseline(args.workload, cycles=max(1, min(args.steps, 8)))
    from tests.oracle import Oracle
    scale = {"bisod3d": 0.25, "sedov3d": 0.125, "sod2d_lagrange": 1.0}[args.workload]
    p = build_params(args.workload, scale)
    o = Oracle(p, cr_pow=False)
    o.init()
    o.iterate(args.warmup)
    t0 = time.perf_counter()
    o.iterate(args.steps)
    dt = time.perf_counter() - t0
    v = p.ncell * args.steps / dt
    base["value"] = v
    base["sample"] = (f"{args.steps} iterations of a {p.nx}x{p.ny}x{p.nz if p.dim == 3 else 1} slab "
                      f"({p.ncell} cells) of the workload; the reference itself needs the Arcane "
                      f"framework and cannot be built here, so its sequential restatement runs")
    out = {"metric": METRIC, "value": v, "unit": "cell-cycles/s", "impl": "reference",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": WORKLOADS[args.workload][0], "cells": p.ncell},
           "cpu_baseline": base,
           "e2e": {"value": v, "unit": "cell-cycles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_ours(args):
    import torch
    import mahyco_b200 as mb
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    lib = mb.load()
    p = build_params(args.workload)
    ncell, nnode = p.ncell, p.nnode
    # -- device-resident throughput
    h = mb.Hydro(p, lib)
    h.hydroStartInit()
    h.cycle(args.warmup)
    st = h.synchronize()
    stream = torch.cuda.ExternalStream(h.stream_handle)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
            torch.cuda.synchronize()

    barrier()
    with ClockSampler(local) as clocks:
        e0.record(stream)
        h.cycle(args.steps)
        e1.record(stream)
        e1.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    st |= h.synchronize()
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    value = world * ncell * args.steps / (ms * 1e-3)
    # -- per-kernel device times (events on the case stream around each group)
    nprof = max(2 * p.dim, min(args.steps, 4 * p.dim))
    stages = h.cycle_timed(nprof)
    s_after = h.scalars()
    h.close()
    # -- end to end through the C ABI: host parameters in, host results out
    import ctypes
    d2h = 0
    t0 = time.perf_counter()
    g = mb.Hydro(p, lib)
    g.hydroStartInit()
    g.cycle(args.warmup)
    for _ in range(args.steps):
        g.cycle(1)
        sc = g.scalars()   # time, deltat, status flags: 40 bytes
        d2h += 40
        if sc["status"] & ~mb.ST_STOP:
            break
    for f in ("Density", "Pressure", "InternalEnergy", "SoundSpeed"):
        d2h += g.field(f).nbytes
    d2h += g.field("Velocity").nbytes
    g.close()
    e2e_s = time.perf_counter() - t0
    e2e_value = world * ncell * args.steps / e2e_s
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    pk = peaks()
    dom = max(stages, key=lambda s: stages[s][0])
    dom_ms, dom_n = stages[dom]
    dom_bytes = stage_bytes(dom, p.dim, p.nb_env, ncell, nnode)
    achieved = dom_bytes / (dom_ms * 1e-3 / dom_n) / 1e9
    traffic = profile_traffic(args.workload).get(dom)
    cycle_bytes = sum(stage_bytes(s, p.dim, p.nb_env, ncell, nnode) * (stages[s][1] / nprof) for s in stages)
    out = {
        "metric": METRIC, "value": value, "unit": "cell-cycles/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload][0], "cells": ncell, "nodes": nnode,
                   "materials": p.nb_env, "remap": bool(p.with_projection),
                   "l2": "working set > 126 MB L2, no flush", "parallelism": f"replicas x{world}"},
        "status": st,
        "gpu_launches": launches_per_cycle(p) * args.steps,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": pk.get("hbm_gbs"),
                     "unit": "GB/s", "frac": achieved / pk.get("hbm_gbs"),
                     "peak_source": "measured" if "how" in pk else "fallback",
                     "traffic": traffic, "algorithmic_bytes_per_launch": dom_bytes,
                     "ms_per_launch": dom_ms / dom_n},
        "cycle_roofline": {"bytes_per_cell_cycle": cycle_bytes / ncell,
                           "achieved_gbs": cycle_bytes * args.steps / (ms * 1e-3) / 1e9 * world},
        "stages_ms_per_cycle": {s: stages[s][0] / nprof for s in stages},
        "clocks": clocks.summary(),
        "e2e": {"value": e2e_value, "unit": "cell-cycles/s",
                "h2d_bytes_per_step": ctypes.sizeof(p) / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                "timer": "host wall clock; includes case allocation, device init, per-iteration status read-back and final field download"},
    }
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args.workload)
    print(json.dumps(out), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="bisod3d", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
