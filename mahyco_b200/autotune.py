"""Autotuner of the run-time launch choices, per mesh-size bucket.

Two choices change how the work of a cycle is laid out on the GPU, never its
arithmetic, so the tuning cycles are ordinary cycles of the run and the
results are bit-identical whatever the tuner picks:

* the layout of the y / z remap sweeps of classical-limiter cases, for
  cells and for nodes: one warp per line (lanes along the sweep), a
  shared-memory tile (coalesced row loads, the warp-per-line arithmetic on
  staged values) or one thread per line chunk (lanes along x, the stencil
  carried in registers).  Which wins depends on the mesh size and the
  number of environments (line chunks per sweep against the device's
  thread slots);
* the grid of every phase's work-list launch: 0 launches one block per work
  item and lets the hardware balance them, k > 0 launches k times the blocks
  the device holds at once, persistent blocks striding over the list (the
  one cross-block reduction, the CFL minimum, is order-independent).

The tuner times each candidate over a few cycles with CUDA events around
every phase (cycle_timed) and installs the fastest per phase.  Decisions
are kept per bucket -- dimension, environments, limiter family and
log2(cells) -- in a JSON cache (MHC_TUNE_CACHE, default
~/.cache/mahyco_b200/tune.json), so the next run of the same bucket installs
them without measuring.

The tile width, the warps per block of the warp-per-line sweeps and the
line-chunk length are template constants of the kernels, fixed at build time
by measurement (mhc_sweep.cuh); the tuner chooses among the compiled layouts.
"""
from __future__ import annotations

import json
import math
import os

CANDIDATES = (0, 1, 2, 4, 8)
LAYOUTS = {1: "warp-per-line", 2: "tile", 3: "line-chunk"}


def cache_path() -> str:
    return os.environ.get("MHC_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "mahyco_b200",
                                                            "tune.json")


def _load() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(key: str, value: dict) -> None:
    data = _load()
    data[key] = value
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path + ".tmp", "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(path + ".tmp", path)
    except OSError:
        pass  # a read-only home: the decision is still installed for this run


def bucket(params_list) -> str:
    """Bucket of a case or of a batch (its cases' total cells): dimension,
    largest number of environments, limiter family (classical limiters 0-2,
    first order, generalised 3-7, pente-borne, third order), log2(cells)."""
    ps = params_list if isinstance(params_list, (list, tuple)) else [params_list]
    cells = sum(p.ncell for p in ps)
    p0 = ps[0]
    if p0.projection_pente_borne:
        fam = "pb"
    elif p0.ordre_projection == 3:
        fam = "o3"
    elif p0.ordre_projection == 1:
        fam = "o1"
    else:
        fam = "lim%d" % p0.projection_limiteur_id if p0.projection_limiteur_id < 3 else "gen"
    return "%dd/ne%d/%s/%s/2^%d" % (p0.dim, max(p.nb_env for p in ps), fam,
                                     "batch%d" % len(ps) if len(ps) > 1 else "case",
                                     int(math.log2(max(1, cells))))


def install(target, decision: dict) -> None:
    target.set_sweep_layout(decision["cell_layout"], decision["node_layout"])
    for stage, scale in decision["grid"].items():
        target.set_stage_grid_scale(stage, scale)


def tune(target, params_list=None, cycles_per_trial: int = 2, candidates=CANDIDATES, use_cache: bool = True) -> dict:
    """Tune a batch (mahyco_b200.Batch) or a case run alone (Hydro) and
    install the fastest choices.  With `params_list` (the cases' parameters)
    and a cached decision for their bucket, that decision is installed
    without measuring.  Otherwise every candidate runs `cycles_per_trial`
    cycles: 3 sweep layouts, then len(candidates) grid scales.  Returns
    {"bucket", "best": {phase: scale}, "cell_layout", "node_layout",
    "ms_per_launch", "cached"}."""
    key = bucket(params_list) if params_list is not None else None
    if use_cache and key is not None:
        hit = _load().get(key)
        if hit:
            install(target, hit)
            return dict(hit, bucket=key, best=hit["grid"], cached=True)
    layout_ms: dict[int, dict[str, float]] = {}
    for lay in LAYOUTS:
        target.set_sweep_layout(lay, lay)
        st = target.cycle_timed(cycles_per_trial)
        layout_ms[lay] = {s: st[s][0] / st[s][1] for s in ("sweep_cells", "sweep_nodes") if st[s][1] > 0}
    def best_layout(stage):
        have = {lay: t[stage] for lay, t in layout_ms.items() if stage in t}
        return min(have, key=have.get) if have else 0
    cell_layout, node_layout = best_layout("sweep_cells"), best_layout("sweep_nodes")
    target.set_sweep_layout(cell_layout, node_layout)
    trials: dict[str, dict[int, float]] = {}
    for cand in candidates:
        target.set_grid_scale(cand)
        st = target.cycle_timed(cycles_per_trial)
        for stage, (ms, n) in st.items():
            if n > 0:
                trials.setdefault(stage, {})[cand] = ms / n
    target.set_grid_scale(0)
    best = {}
    for stage, t in trials.items():
        best[stage] = min(t, key=t.get)
        target.set_stage_grid_scale(stage, best[stage])
    decision = {"cell_layout": cell_layout, "node_layout": node_layout, "grid": best,
                "layout_ms_per_launch": {LAYOUTS[k]: v for k, v in layout_ms.items()}}
    if key is not None:
        _store(key, decision)
    return dict(decision, bucket=key, best=best, ms_per_launch=trials, cached=False)
