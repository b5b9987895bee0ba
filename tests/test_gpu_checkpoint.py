"""Checkpoint / restart of the device-resident state (protection-reprise):
continuing from a checkpoint is bit-identical to never having stopped, in a
fresh case and in the same case after it ran on; mismatched buffers are
refused."""
import numpy as np
import pytest

import mahyco_b200 as mb
from mahyco_b200.cases import PARITY_CASES

pytestmark = pytest.mark.gpu

FIELDS = ("Density", "Pressure", "InternalEnergy", "Velocity", "NodeCoord", "CellMass")


@pytest.mark.parametrize("name", ["adi3d_bisod_superbee", "adi2d_sedov", "lag2d_bar_impact"])
def test_restart_is_bit_identical(name):
    build, _ = PARITY_CASES[name]
    p = build()
    a = mb.Hydro(p)
    a.hydroStartInit()
    a.cycle(7)
    ck = a.checkpoint()
    a.cycle(11)
    ref = {f: a.field(f) for f in FIELDS}
    ref_s = a.scalars()
    # a fresh case continues from the checkpoint
    b = mb.Hydro(p)
    b.hydroStartInit()
    b.restore(ck)
    b.cycle(11)
    for f in FIELDS:
        np.testing.assert_array_equal(b.field(f), ref[f], err_msg=f)
    assert b.scalars() == ref_s
    # the original case goes back and redoes the same iterations
    a.restore(ck)
    a.cycle(11)
    for f in FIELDS:
        np.testing.assert_array_equal(a.field(f), ref[f], err_msg=f)
    a.close()
    b.close()


def test_restore_refuses_other_cases():
    b1, _ = PARITY_CASES["adi2d_sedov"]
    b2, _ = PARITY_CASES["adi2d_two_state_vanleer"]
    a = mb.Hydro(b1())
    a.hydroStartInit()
    ck = a.checkpoint()
    c = mb.Hydro(b2())
    c.hydroStartInit()
    with pytest.raises(mb.MahycoError):
        c.restore(ck)
    with pytest.raises(mb.MahycoError):
        a.restore(ck[:-8])
    a.close()
    c.close()


def test_async_scalars_match_synchronous():
    build, _ = PARITY_CASES["adi2d_sedov"]
    h = mb.Hydro(build())
    h.hydroStartInit()
    seen = []
    prev = None
    for _ in range(6):
        h.cycle(1)
        slot = h.scalars_request()
        if prev is not None:
            seen.append(h.scalars_wait(prev))
        prev = slot
    seen.append(h.scalars_wait(prev))
    assert [s["iteration"] for s in seen] == [1, 2, 3, 4, 5, 6]
    assert seen[-1] == h.scalars()
    h.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["adi3d_bisod_superbee", "adi2d_sedov", "lag2d_sod_mono"])
def test_graph_replay_matches_plain_launches(name):
    """The CUDA-graph path (captured once without running, n = 0, then
    replayed per 6-iteration period) gives the plain launches' fields bitwise."""
    from mahyco_b200 import Hydro
    from mahyco_b200.cases import PARITY_CASES
    build, n = PARITY_CASES[name]
    out = []
    for graph in (False, True):
        h = Hydro(build())
        h.hydroStartInit()
        if graph:
            h.cycle(0, graph=True)
        h.cycle(5, graph=graph)
        h.cycle(n - 5, graph=graph)
        assert h.synchronize() == 0
        out.append({f: h.field(f) for f in ("Density", "Pressure", "InternalEnergy", "Velocity")} |
                   {"scalars": np.array([h.scalars()["time"], h.scalars()["deltat"]])})
        h.close()
    for f in out[0]:
        assert np.array_equal(out[0][f], out[1][f]), f
