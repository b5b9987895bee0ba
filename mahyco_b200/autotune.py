"""Launch-shape autotuner for batched runs.

Every kernel phase of the engine walks a work list of (case, virtual block)
items.  Its launch shape is a grid scale: 0 launches one block per work item
and lets the hardware block scheduler balance them; k > 0 launches k times
the number of blocks the device holds at once, and those persistent blocks
stride over the list.  Which one wins depends on the phase (register and
shared-memory footprint, work per item) and on the mix of case sizes, so the
tuner measures it on the live batch: for each candidate it runs a few cycles
with CUDA events around every phase, then keeps the fastest candidate per
phase.

A launch shape only changes which block processes which work item, never
the arithmetic (the one cross-block reduction, the CFL minimum, is an
order-independent minimum), so the tuning cycles are ordinary cycles of the
run and the results are bit-identical whatever the tuner picks.
"""
from __future__ import annotations

CANDIDATES = (0, 1, 2, 4, 8)


def tune(batch, cycles_per_trial: int = 2, candidates=CANDIDATES) -> dict:
    """Time each candidate grid scale on `batch` and install the fastest per
    phase.  Advances every active case by len(candidates) * cycles_per_trial
    iterations.  Returns {"best": {phase: scale}, "ms_per_launch": {phase:
    {scale: ms}}}."""
    trials: dict[str, dict[int, float]] = {}
    for cand in candidates:
        batch.set_grid_scale(cand)
        st = batch.cycle_timed(cycles_per_trial)
        for stage, (ms, n) in st.items():
            if n > 0:
                trials.setdefault(stage, {})[cand] = ms / n
    batch.set_grid_scale(0)
    best = {}
    for stage, t in trials.items():
        best[stage] = min(t, key=t.get)
        batch.set_stage_grid_scale(stage, best[stage])
    return {"best": best, "ms_per_launch": trials}
