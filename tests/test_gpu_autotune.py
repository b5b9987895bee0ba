"""The tuner's choices never change results: every y / z sweep layout
(warp per line, shared-memory tile, line chunks) and any tuned launch grid
give bit-identical fields, and a tuned run equals an untuned one; decisions
are cached per mesh-size bucket and installed from the cache."""
import numpy as np
import pytest

FIELDS = ("Density", "Pressure", "InternalEnergy", "Velocity", "NodeMass")


def _run(p, cycles, layout=None, tune_kw=None):
    import mahyco_b200 as mb
    from mahyco_b200.autotune import tune
    h = mb.Hydro(p)
    h.hydroStartInit()
    info = None
    if layout is not None:
        h.set_sweep_layout(layout, layout)
    if tune_kw is not None:
        info = tune(h, params_list=p, **tune_kw)
    done = h.scalars()["iteration"]
    h.cycle(cycles - done)
    assert h.synchronize() == 0
    out = {f: h.field(f) for f in FIELDS}
    out["scalars"] = h.scalars()
    h.close()
    return out, info


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["bisod3d", "sedov2d"])
def test_every_sweep_layout_gives_the_same_bits(case):
    from mahyco_b200.cases import sod, sedov, SUPERBEE
    p = (sod(dim=3, n=(32, 12, 10), L=(1.0, 0.3, 0.25), bi=True, limiter=SUPERBEE, deltat_init=1e-3)
         if case == "bisod3d" else sedov(dim=2, n=(40, 40), deltat_init=1e-4))
    ref, _ = _run(p, 30, layout=0)
    for lay in (1, 2, 3):
        got, _ = _run(p, 30, layout=lay)
        for f in FIELDS:
            assert np.array_equal(got[f], ref[f]), (lay, f)
        assert got["scalars"] == ref["scalars"]


@pytest.mark.gpu
def test_tuned_run_equals_untuned_and_is_cached(tmp_path, monkeypatch):
    from mahyco_b200.cases import sod, SUPERBEE
    monkeypatch.setenv("MHC_TUNE_CACHE", str(tmp_path / "tune.json"))
    p = sod(dim=3, n=(48, 12, 12), L=(1.0, 0.25, 0.25), bi=True, limiter=SUPERBEE, deltat_init=1e-3)
    ref, _ = _run(p, 40)
    got, info = _run(p, 40, tune_kw=dict(cycles_per_trial=1, use_cache=True))
    assert not info["cached"] and info["cell_layout"] in (1, 2, 3) and info["node_layout"] in (1, 2, 3)
    for f in FIELDS:
        assert np.array_equal(got[f], ref[f]), f
    again, info2 = _run(p, 40, tune_kw=dict(cycles_per_trial=1, use_cache=True))
    assert info2["cached"] and info2["bucket"] == info["bucket"]
    assert (info2["cell_layout"], info2["node_layout"], info2["best"]) == (info["cell_layout"], info["node_layout"],
                                                                            info["best"])
    for f in FIELDS:
        assert np.array_equal(again[f], ref[f]), f
