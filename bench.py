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
    "batch2d": ("batched: 4096 independent 2D Sod/BiSod cases, sides log-uniform 32..512, seeded states, "
                "ADI remap, vanleer, FP64", 2),
    "serve": ("served: Poisson arrivals of mixed 2D/3D Sedov, 3D BiSod, stiffened-gas water/air and "
              "Mie-Gruneisen bar impact requests of 1e3..1e7 cells, HBM-budget admission, continuous "
              "batching, FP64", 2),
}


def build_params(name: str, scale: float = 1.0):
    from mahyco_b200.cases import workload
    return workload(name, scale)


# algorithmic bytes per launch of each kernel group: compulsory traffic of
# the live fields (one read and/or write of each per pass, FP64)
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


def max_over_ranks(ms: float, device: str = "cuda") -> float:
    """Slowest rank's time (all ranks take this collective in the same
    order); the identity without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return ms
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank: float, world: int, ms_max: float) -> float:
    """Whole-job throughput of `world` replicas: all ranks' units over the
    slowest rank's time."""
    return world * units_per_rank / (ms_max * 1e-3)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms.  Entering
    waits for nvidia-smi's first sample (its start-up takes driver locks and
    must not overlap the timed region); the summary keeps the samples taken
    after that, and leaving waits for at least one of them."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.first = 0
        self.proc = None

    def _wait(self, n: int, limit: float):
        t0 = time.perf_counter()
        while len(self.samples) <= n and time.perf_counter() - t0 < limit and self.proc.poll() is None:
            time.sleep(0.005)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            self._wait(0, 10.0)
        except OSError:
            self.proc = None
        self.first = len(self.samples)
        return self

    def _read(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 8:
                self.samples.append(f)

    def __exit__(self, *a):
        if self.proc:
            self._wait(self.first, 1.0)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        samples = self.samples[self.first:]
        if not samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in samples for i in range(4) if s[4 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(samples)}


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


def _oracle_slab(workload: str, cells_target: float):
    """A slab of the workload with the same cell size and about
    `cells_target` cells (the CPU sample of the reference arm)."""
    full = build_params(workload)
    return build_params(workload, min(1.0, (cells_target / full.ncell) ** (1.0 / full.dim)))


def _oracle_worker(task):
    """One host core: the CPU oracle on its own slab, timed after warm-up
    (spawned process; returns cell-cycles and seconds)."""
    workload, cells_target, warmup, steps, seed = task
    sys.path.insert(0, ROOT)
    from tests.oracle import Oracle
    if workload == "batch2d":
        import random
        from mahyco_b200.cases import seeded_two_state
        rng = random.Random(seed)
        cases = []
        while sum(c.ncell for c in cases) < cells_target:
            cases.append(seeded_two_state(seed * 7919 + len(cases), rng.randint(32, 96)))
    else:
        cases = [_oracle_slab(workload, cells_target)]
    work, sec = 0, 0.0
    for p in cases:
        o = Oracle(p, cr_pow=False)
        o.init()
        o.iterate(warmup)
        t0 = time.perf_counter()
        o.iterate(steps)
        sec += time.perf_counter() - t0
        work += p.ncell * steps
    return work, sec, sum(c.ncell for c in cases)


def oracle_throughput(workload: str, steps: int, warmup: int, cores: int | None = None,
                      cell_cycles_per_core: float = 8e6) -> dict:
    """The CPU oracle (sequential restatement of the reference path) on
    every host core at once, one independent slab per core; aggregate
    cell-cycles/s over the parallel phase."""
    import multiprocessing as mp
    cores = cores or len(os.sched_getaffinity(0))
    wl = "bisod3d" if workload == "serve" else workload
    cells_target = max(2000.0, cell_cycles_per_core / max(1, steps))
    tasks = [(wl, cells_target, warmup, steps, 1000 + r) for r in range(cores)]
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.map(_oracle_worker, tasks)
    wall = time.perf_counter() - t0
    work = sum(r[0] for r in res)
    slowest = max(r[1] for r in res)
    return {"value": work / slowest, "unit": "cell-cycles/s", "cores": cores, "kind": "port",
            "sample": f"{cores} independent {'sets of seeded 2D cases' if wl == 'batch2d' else 'slabs'} of "
                      f"about {int(res[0][2])} cells of the {wl} workload (same cell size and states), "
                      f"{steps} timed iterations each after {warmup} warm-up, one spawned process per host "
                      f"core running the sequential oracle; value = all cores' cell-cycles / slowest core's "
                      f"time (wall {wall:.1f} s including start-up)"}


def cpu_baseline(workload: str, steps: int = 20) -> dict:
    """Bounded CPU sample reported beside the GPU number (about 10 s)."""
    return oracle_throughput(workload, steps=steps, warmup=1)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    base = oracle_throughput(args.workload, steps=args.steps, warmup=max(1, args.warmup))
    base["sample"] += ("; the reference itself needs the Arcane framework and cannot be built here, so "
                       "its sequential CPU restatement (oracle/) runs")
    v = base["value"]
    out = {"metric": METRIC, "value": v, "unit": "cell-cycles/s", "impl": "reference",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": WORKLOADS[args.workload][0]},
           "cpu_baseline": base,
           "e2e": {"value": v, "unit": "cell-cycles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def measure_plain(lib, p, steps: int, warmup: int, local: int = 0, world: int = 1) -> dict:
    """The plain form on one case, device-resident: W warm-up iterations,
    then K iterations replayed from the case's CUDA graph (captured before
    the warm-up) between CUDA events on the case stream; then per-kernel
    device times (events around every kernel group) for the roofline."""
    import torch
    import mahyco_b200 as mb
    from mahyco_b200.autotune import tune
    h = mb.Hydro(p, lib)
    h.hydroStartInit()
    # the plain form at its best: sweep layouts and launch grids tuned for
    # this mesh-size bucket (or installed from the tuning cache); the
    # tuning cycles are part of the warm-up
    tuned = tune(h, params_list=p, cycles_per_trial=1)
    h.cycle(0, graph=True)  # capture the CUDA graph of one sweep-order period (no iteration)
    h.cycle(warmup, graph=True)
    st = h.synchronize()
    stream = torch.cuda.ExternalStream(h.stream_handle)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
            torch.cuda.synchronize()

    barrier()
    l0 = h.launches
    with ClockSampler(local) as clocks:
        e0.record(stream)
        h.cycle(steps, graph=True)
        e1.record(stream)
        e1.synchronize()
    barrier()
    launches = h.launches - l0
    ms = e0.elapsed_time(e1)
    st |= h.synchronize()
    ms = max_over_ranks(ms)
    nprof = max(2 * p.dim, min(steps, 4 * p.dim))
    stages = h.cycle_timed(nprof)
    h.close()
    ncell, nnode = p.ncell, p.nnode
    pk = peaks()
    dom = max(stages, key=lambda s: stages[s][0])
    dom_ms, dom_n = stages[dom]
    dom_bytes = stage_bytes(dom, p.dim, p.nb_env, ncell, nnode)
    achieved = dom_bytes / (dom_ms * 1e-3 / dom_n) / 1e9
    cycle_bytes = sum(stage_bytes(s, p.dim, p.nb_env, ncell, nnode) * (stages[s][1] / nprof) for s in stages)
    return {
        "value": replica_value(ncell * steps, world, ms), "ms_per_step": ms / steps, "status": st,
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": pk.get("hbm_gbs"),
                     "unit": "GB/s", "frac": achieved / pk.get("hbm_gbs"),
                     "peak_source": "measured" if "how" in pk else "fallback",
                     "algorithmic_bytes_per_launch": dom_bytes, "ms_per_launch": dom_ms / dom_n},
        "cycle_roofline": {"bytes_per_cell_cycle": cycle_bytes / ncell,
                           "achieved_gbs": cycle_bytes * steps / (ms * 1e-3) / 1e9 * world},
        "stages_ms_per_cycle": {s: stages[s][0] / nprof for s in stages},
        "clocks": clocks.summary(),
        "autotune": {k: tuned[k] for k in ("bucket", "cell_layout", "node_layout", "best", "cached")},
    }


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
    parts = {}
    w0 = time.perf_counter()
    # -- device-resident throughput of the plain form
    m = measure_plain(lib, p, args.steps, args.warmup, local, world)
    m["roofline"]["traffic"] = profile_traffic(args.workload).get(m["roofline"]["kernel"])
    parts["plain"] = time.perf_counter() - w0
    # -- end to end through the C ABI: host parameters in, host results out
    # (into page-locked result buffers the job allocates once, up front)
    import ctypes
    d2h = 0
    e2e_fields = ("Density", "Pressure", "InternalEnergy", "SoundSpeed", "Velocity")
    e2e_out = {f: torch.empty(3 * nnode if f == "Velocity" else ncell, dtype=torch.float64,
                              pin_memory=True).numpy() for f in e2e_fields}
    t0 = time.perf_counter()
    g = mb.Hydro(p, lib)
    g.hydroStartInit()
    # the iterations go in periods of 6 through the case's CUDA graph
    # (mhc_cycle_graph, captured on the first period inside the timed
    # region); after every period its status (time, deltat, iteration,
    # flags) comes back to the host, the read of period k overlapping
    # period k+1 on the GPU
    prev = None
    done = 0
    while done < args.steps:
        n = min(6, args.steps - done)
        g.cycle(n, graph=True)
        done += n
        slot = g.scalars_request()
        d2h += 96  # the case's scalars record
        if prev is not None and g.scalars_wait(prev)["status"] & ~mb.ST_STOP:
            break
        prev = slot
    if prev is not None:
        g.scalars_wait(prev)
    for f in e2e_fields:
        d2h += g.field(f, out=e2e_out[f]).nbytes
    g.close()
    e2e_s = time.perf_counter() - t0
    e2e_value = world * ncell * args.steps / e2e_s
    parts["e2e"] = e2e_s
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    out = {
        "metric": METRIC, "value": m["value"], "unit": "cell-cycles/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload][0], "cells": ncell, "nodes": nnode,
                   "materials": p.nb_env, "remap": bool(p.with_projection),
                   "l2": "working set > 126 MB L2, no flush", "parallelism": f"replicas x{world}",
                   "timing": "K iterations replayed from the case's CUDA graph of one 6-iteration period"},
        "status": m["status"],
        "gpu_launches": m["gpu_launches"],
        "roofline": m["roofline"],
        "cycle_roofline": m["cycle_roofline"],
        "stages_ms_per_cycle": m["stages_ms_per_cycle"],
        "autotune": m["autotune"],
        "clocks": m["clocks"],
        "e2e": {"value": e2e_value, "unit": "cell-cycles/s",
                "h2d_bytes_per_step": ctypes.sizeof(p) / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                "timer": "host wall clock; includes case allocation, device init, the graph capture, the status read-back after every 6-iteration period (overlapping the next period) and the final field download into page-locked result buffers allocated before the timed region"},
    }
    if world == 1 and not args.no_extras:
        # the other stated configurations, each at its stated size:
        # 3D Sedov 384^3 (the plain form's roofline target), the batched
        # form on 4096 2D cases x 100 cycles and the served form on the
        # mixed request stream, both against the plain form
        w0 = time.perf_counter()
        sp = build_params("sedov3d")
        sm = measure_plain(lib, sp, steps=10, warmup=3, local=local)
        out["sedov3d"] = dict(sm, workload=WORKLOADS["sedov3d"][0], cells=sp.ncell, steps=10, warmup=3,
                              unit="cell-cycles/s")
        parts["sedov3d"] = time.perf_counter() - w0
        w0 = time.perf_counter()
        sub = argparse.Namespace(**vars(args))
        sub.workload, sub.cases, sub.steps, sub.warmup, sub.plain_sample = "bisod3d", 4096, 100, 0, 512
        bo = run_batch(sub)
        out["batched"] = {"value": bo["value"], "plain_value": bo["plain"]["value"],
                          "batched_vs_plain": bo["batched_vs_plain"], "same_results": bo["plain"]["same_results"],
                          "ms_per_step": bo["ms_per_step"], "latency_s": bo["latency_s"],
                          "plain_latency_s": bo["plain"]["latency_s"],
                          "config": f"{sub.cases} cases of the batch2d workload ({bo['config']['cells']} cells), "
                                    f"{sub.steps} timed cycles each; plain form through each case's own CUDA "
                                    f"graph on every {sub.cases // sub.plain_sample}-th case "
                                    f"({bo['plain']['sample_cases']} cases)",
                          "autotune": bo["autotune"], "gpu_launches": bo["gpu_launches"], "clocks": bo["clocks"]}
        parts["batched"] = time.perf_counter() - w0
        # the served form at two stated Poisson rates: 16/s (about half of
        # the plain form's capacity: the latency regime) and 64/s (above
        # it: both forms run flat out, the throughput regime)
        for key, rate in (("served", 16.0), ("served_overload", 64.0)):
            w0 = time.perf_counter()
            sub = argparse.Namespace(**vars(args))
            sub.workload, sub.requests, sub.rate, sub.steps, sub.cycles_per_step = "bisod3d", 120, rate, 30, 4
            so = run_serve(sub)
            out[key] = {"value": so["value"], "plain_value": so["plain"]["value"],
                        "served_vs_plain": so["served_vs_plain"], "latency_s": so["latency_s"],
                        "plain_latency_s": so["plain"]["latency_s"], "latency_by_class_s": so["latency_by_class_s"],
                        "plain_busy_value": so["plain"]["busy_value"], "failed": len(so["failed"]),
                        "offered_cell_cycles_per_s": so["config"]["offered_cell_cycles_per_s"],
                        "work_share_requests_ge_1e6_cells": so["work_share_requests_ge_1e6_cells"],
                        "config": f"{sub.requests} requests of the serve mix (1e3..1e7 cells) at a Poisson "
                                  f"rate of {sub.rate}/s, {sub.steps} iterations each",
                        "gpu_launches": so["gpu_launches"], "clocks": so["clocks"]}
            parts[key] = time.perf_counter() - w0
    if world == 1 and not args.no_cpu_baseline:
        w0 = time.perf_counter()
        out["cpu_baseline"] = cpu_baseline(args.workload)
        parts["cpu_baseline"] = time.perf_counter() - w0
    out["parts_wall_s"] = parts
    print(json.dumps(out), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def batch_cases(count: int, seed: int = 2024):
    from mahyco_b200.cases import seeded_two_state, log_uniform_sides
    sides = log_uniform_sides(count, seed=seed)
    return [seeded_two_state(seed * 100003 + i, n) for i, n in enumerate(sides)]


def run_batch(args):
    """Batched form: every case resident, one launch per phase for all of
    them, cycles replayed from a CUDA graph, launch shapes autotuned during
    the warm-up; against the plain form (one case at a time through its own
    handle) on a seeded sample of the same cases."""
    import ctypes
    import torch
    import mahyco_b200 as mb
    from mahyco_b200.autotune import tune, CANDIDATES
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    lib = mb.load()
    all_cases = batch_cases(args.cases)
    # N > 1: the cases are shared between the ranks by device bytes (every
    # case on exactly one GPU; no exchange while they run)
    from mahyco_b200.partition import partition_by_bytes, gather_results
    sizes = [lib.mhc_case_device_bytes(ctypes.byref(p)) for p in all_cases]
    mine = partition_by_bytes(sizes, world)[rank]
    cases = [all_cases[i] for i in mine]
    tune_cycles = 2 * (len(CANDIDATES) + 3)
    warm = max(args.warmup, tune_cycles + 4)
    limit = warm + args.steps
    cells = sum(p.ncell for p in cases)
    total_cells = sum(p.ncell for p in all_cases)
    # -- batched arm
    t_wall0 = time.perf_counter()
    b = mb.Batch(lib)
    idx = [b.add(p, iteration_limit=limit) for p in cases]
    b.init()
    tuned = tune(b, params_list=cases, cycles_per_trial=2)
    if tuned["cached"]:  # installed without measuring: run the cycles the trials would have run
        b.cycle(tune_cycles)
    st = b.cycle_timed(2)  # per-phase device time with the tuned shapes
    stages = {k: v[0] / 2 for k, v in st.items()}
    b.cycle(warm - tune_cycles - 2, graph=True)
    b.synchronize()
    stream = torch.cuda.ExternalStream(b.stream_handle)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    l0 = b.launches
    with ClockSampler(local) as clocks:
        e0.record(stream)
        b.cycle(args.steps, graph=True)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    launches = b.launches - l0
    done = [b.scalars(i) for i in idx]
    t_wall = max_over_ranks((time.perf_counter() - t_wall0) * 1e3) * 1e-3
    bad = sum(1 for d in done if d["iteration"] != limit)
    ms = max_over_ranks(ms)
    # whole job: every rank's cells over the slowest rank's device time
    batched = total_cells * args.steps / (ms * 1e-3)
    # every case's final (iteration, time) gathered on rank 0
    gathered = gather_results({mine[j]: (done[j]["iteration"], done[j]["time"]) for j in range(len(mine))}, world)
    # -- plain arm on a seeded sample (every k-th case), device time of the
    # same K cycles per case, plus its per-solve wall latency
    k = max(1, len(cases) // args.plain_sample) if args.plain_sample > 0 else 1
    sample = list(range(0, len(cases), k))
    plain_ms, plain_cells, lat, same, plain_launches = 0.0, 0, [], True, 0
    check = set(sample[:: max(1, len(sample) // 8)])
    for i in sample:
        p = cases[i]
        w0 = time.perf_counter()
        h = mb.Hydro(p, lib)
        h.hydroStartInit()
        h.cycle(0, graph=True)  # the plain form at its best: its own CUDA graph
        h.cycle(warm, graph=True)
        st = torch.cuda.ExternalStream(h.stream_handle)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(st)
        pl0 = h.launches
        h.cycle(args.steps, graph=True)
        plain_launches += h.launches - pl0
        a1.record(st)
        a1.synchronize()
        rho = h.field("Density")
        lat.append(time.perf_counter() - w0)
        plain_ms += a0.elapsed_time(a1)
        plain_cells += p.ncell
        if i in check:
            import numpy as np
            same &= bool(np.array_equal(rho, b.field(idx[i], "Density")))
        h.close()
    b.close()
    plain = plain_cells * args.steps / (plain_ms * 1e-3)
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([plain_cells * args.steps, plain_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t)  # the sampled plain solves of all ranks (each rank's GPU runs its own)
        plain = world * float(t[0]) / (float(t[1]) * 1e-3)
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    lat.sort()
    out = {
        "metric": METRIC, "value": batched, "unit": "cell-cycles/s", "n_gpus": world,
        "steps": args.steps, "warmup": warm, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOADS["batch2d"][0], "cases": len(all_cases), "cells": total_cells,
                   "step": "one cycle of every case", "graph": "CUDA graph of 6 cycles",
                   "l2": "working set > 126 MB L2, no flush",
                   "parallelism": f"cases shared by device bytes over {world} GPU(s)" if world > 1 else "1 GPU",
                   "cases_gathered": len(gathered) if gathered is not None else None},
        "batched_vs_plain": batched / plain,
        "plain": {"value": plain, "unit": "cell-cycles/s", "sample_cases": len(sample),
                  "sample_cells": plain_cells, "same_results": same, "gpu_launches": plain_launches,
                  "latency_s": {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))]},
                  "how": "each sampled case alone through its own handle: create, init, capture of its CUDA "
                         "graph, warm-up, K timed cycles replayed from the graph"},
        "latency_s": {"p50": t_wall, "p99": t_wall,
                      "how": "every case of the batch completes with the batch: host wall clock from the first "
                             "case creation to the last status read-back"},
        "autotune": {k: tuned[k] for k in ("bucket", "cell_layout", "node_layout", "best", "cached")},
        "stages_ms_per_cycle": stages,
        "cases_not_at_limit": bad,
        "gpu_launches": launches,
        "clocks": clocks.summary(),
        "e2e": {"value": total_cells * args.steps / t_wall, "unit": "cell-cycles/s",
                "h2d_bytes_per_step": len(cases) * ctypes.sizeof(cases[0]) / args.steps,
                "d2h_bytes_per_step": len(cases) * 40 / args.steps,
                "timer": "host wall clock of the whole batched run: case creation, init, tuning, warm-up, K cycles, status read-back"},
    }
    if args.workload == "batch2d":
        print(json.dumps(out), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return out


def serve_requests(count: int, seed: int = 7):
    """(kind, params, iterations) of the served mix: kinds uniform, cells
    log-uniform in [1e3, 1e7] (the bar impact is always 80x400)."""
    import math
    import random
    from mahyco_b200.cases import serving_request, SERVING_KINDS
    rng = random.Random(seed)
    out = []
    for _ in range(count):
        kind = rng.choice(SERVING_KINDS)
        cells = int(math.exp(rng.uniform(math.log(1e3), math.log(1e7))))
        out.append((kind, serving_request(kind, cells)))
    return out


def run_serve(args):
    """Served form: a request loop (mhc_server_*) fed by Poisson arrivals,
    against sequential plain solves of the same requests on the same GPU."""
    import random
    import torch
    import mahyco_b200 as mb
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1 and not torch.distributed.is_initialized():
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    lib = mb.load()
    its = args.steps
    all_reqs = serve_requests(args.requests)
    rng = random.Random(11)
    all_arrivals, t = [], 0.0
    for _ in all_reqs:
        t += rng.expovariate(args.rate)
        all_arrivals.append(t)
    # N > 1: the request stream is shared between the GPUs by device bytes
    # (each rank serves its requests at their arrival times)
    import ctypes
    from mahyco_b200.partition import partition_by_bytes, gather_results
    mine = partition_by_bytes([lib.mhc_case_device_bytes(ctypes.byref(p)) for _, p in all_reqs], world)[rank]
    reqs = [all_reqs[i] for i in mine]
    arrivals = [all_arrivals[i] for i in mine]
    work = sum(p.ncell for _, p in reqs) * its
    total_work = sum(p.ncell for _, p in all_reqs) * its
    # warm-up: one small solve of every kind through the server (module load,
    # pools, first launches)
    srv = mb.Server()
    for kind, p in serve_requests(len(reqs))[:10]:
        if p.ncell < 50000:
            srv.submit(p, 3)
    while srv.stats()["queued"] or srv.stats()["running"]:
        srv.step(3)
    srv.close()
    srv = mb.Server()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    nxt, tickets, done_at = 0, {}, {}
    l0 = srv.launches
    with ClockSampler(local) as clocks:
        while len(done_at) < len(reqs):
            now = time.perf_counter() - t0
            while nxt < len(reqs) and arrivals[nxt] <= now:
                tickets[srv.submit(reqs[nxt][1], its)] = nxt
                nxt += 1
            if not tickets or len(done_at) == len(tickets):
                if nxt < len(reqs):
                    time.sleep(max(0.0, min(0.002, arrivals[nxt] - now)))
                continue
            srv.step(args.cycles_per_step)
            now = time.perf_counter() - t0
            for tk in srv.take_completed():
                i = tickets[tk]
                st = srv.poll(tk)
                done_at[i] = (now, st["state"], st["status"])
                srv.release(tk)
    launches = srv.launches - l0
    srv.close()
    # whole job: every rank's work over the latest completion (from the
    # stream's first arrival) of any rank
    makespan = max(d[0] for d in done_at.values()) - all_arrivals[0]
    makespan = max_over_ranks(makespan * 1e3) * 1e-3
    lat_local = {mine[i]: done_at[i][0] - arrivals[i] for i in range(len(reqs))}
    failed = [{"kind": reqs[i][0], "cells": reqs[i][1].ncell, "status": d[2]}
              for i, d in sorted(done_at.items()) if d[1] != mb.REQ_DONE]
    served = total_work / makespan
    # sequential plain solves, each alone: create, init, cycles, read-back
    service = []
    for kind, p in reqs:
        # the plain form at its best: each request solved both with plain
        # launches and with its own CUDA graph of one sweep-order period
        # (capture included), the faster kept
        best = None
        for graph in (False, True):
            w0 = time.perf_counter()
            h = mb.Hydro(p, lib)
            h.hydroStartInit()
            h.cycle(its, graph=graph)
            h.scalars()
            h.close()
            dt_s = time.perf_counter() - w0
            best = dt_s if best is None else min(best, dt_s)
        service.append(best)
    fin, plat_local = 0.0, {}
    for j, (a, sv) in enumerate(zip(arrivals, service)):  # FIFO queue under the same arrivals
        fin = max(fin, a) + sv
        plat_local[mine[j]] = fin - a
    # both forms over the same arrivals: work / (last completion - first arrival)
    plain = total_work / (max_over_ranks((fin - all_arrivals[0]) * 1e3) * 1e-3)
    busy = max_over_ranks(sum(service) * 1e3) * 1e-3
    # every request's latency in both forms, gathered on rank 0
    g_lat = gather_results(lat_local, world)
    g_plat = gather_results(plat_local, world)
    g_fail = gather_results({rank: failed}, world)
    if rank != 0:
        return None
    lat = sorted(g_lat.values())
    plat = sorted(g_plat.values())
    failed = [f for r in sorted(g_fail) for f in g_fail[r]]
    reqs, arrivals, work = all_reqs, all_arrivals, total_work

    def pct(v, q):
        return v[min(len(v) - 1, int(q * len(v)))]

    # latency by size class (the server's classes: < 3e4, < 1e6, larger)
    def cls_of(n):
        return "small" if n < 30000 else ("medium" if n < 1000000 else "large")
    by_cls = {}
    for i, (_, p) in enumerate(reqs):
        c = cls_of(p.ncell)
        by_cls.setdefault(c, ([], []))
        by_cls[c][0].append(g_lat[i])
        by_cls[c][1].append(g_plat[i])
    cls_lat = {c: {"requests": len(v[0]), "served_p50": pct(sorted(v[0]), 0.5), "served_p99": pct(sorted(v[0]), 0.99),
                   "plain_p50": pct(sorted(v[1]), 0.5), "plain_p99": pct(sorted(v[1]), 0.99)}
               for c, v in sorted(by_cls.items())}
    big = sum(p.ncell for _, p in reqs if p.ncell >= 1000000) * its
    out = {
        "metric": METRIC, "value": served, "unit": "cell-cycles/s", "n_gpus": world,
        "steps": its, "warmup": 3, "ms_per_step": None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOADS["serve"][0], "requests": len(reqs), "rate_per_s": args.rate,
                   "parallelism": f"requests shared by device bytes over {world} GPU(s)" if world > 1 else "1 GPU",
                   "iterations_per_request": its, "cells": sum(p.ncell for _, p in reqs),
                   "cycles_per_step": args.cycles_per_step,
                   "offered_cell_cycles_per_s": work / (arrivals[-1] - arrivals[0]),
                   "l2": "mixed sizes; large requests exceed L2"},
        "latency_s": {"p50": pct(lat, 0.5), "p99": pct(lat, 0.99), "max": lat[-1]},
        "latency_by_class_s": cls_lat,
        "work_share_requests_ge_1e6_cells": big / work,
        "failed": failed,
        "served_vs_plain": served / plain,
        "plain": {"value": plain, "unit": "cell-cycles/s",
                  "latency_s": {"p50": pct(plat, 0.5), "p99": pct(plat, 0.99), "max": plat[-1]},
                  "busy_value": total_work / busy,
                  "how": "the same requests solved one after another through their own handles (create, init, "
                         "iterations, status read-back), each timed with plain launches and with its own CUDA "
                         "graph and the faster kept; value and latency from a FIFO queue of those service times "
                         "under the same arrivals; busy_value = work / sum of service times"},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
        "e2e": {"value": served, "unit": "cell-cycles/s",
                "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "timer": "host wall clock from the first arrival to the last completion"},
    }
    if args.workload == "serve":
        print(json.dumps(out), flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="bisod3d", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="plain workloads: skip the batched and served samples")
    ap.add_argument("--kernels-only", action="store_true",
                    help="run init, W and K cycles of one case and exit (for ncu launch lists)")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="with --kernels-only: linear scale of the mesh (same cell size)")
    ap.add_argument("--cases", type=int, default=4096, help="batch2d: number of cases")
    ap.add_argument("--plain-sample", type=int, default=0,
                    help="batch2d: cases timed one at a time (0 = all of them)")
    ap.add_argument("--requests", type=int, default=120, help="serve: number of requests")
    ap.add_argument("--rate", type=float, default=8.0, help="serve: Poisson arrival rate (1/s)")
    ap.add_argument("--cycles-per-step", type=int, default=4, help="serve: cycles between admissions")
    args = ap.parse_args()
    if args.kernels_only:
        import mahyco_b200 as mb
        h = mb.Hydro(build_params(args.workload, args.scale))
        h.hydroStartInit()
        h.cycle(args.warmup + args.steps)
        print(json.dumps({"kernels_only": args.workload, "scale": args.scale, "cells": h.ncell,
                          "launches": h.launches, "scalars": h.scalars()}))
        h.close()
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch2d":
        run_batch(args)
    elif args.workload == "serve":
        run_serve(args)
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
