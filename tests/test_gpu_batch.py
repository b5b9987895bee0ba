"""Batched execution: many cases of uneven sizes and kinds in one batch.

Each case of a batch must give the same fields, bit for bit, as the same
case run alone (which is itself bit-identical to the oracle, see
test_gpu_parity.py), with plain launches and with the CUDA-graph replay; a
case that fails or stops inside a batch must not disturb its neighbours.
"""
import numpy as np
import pytest

from mahyco_b200.cases import PARITY_CASES, seeded_two_state

FIELDS = ["Density", "Pressure", "InternalEnergy", "SoundSpeed", "PseudoViscosity", "CellMass",
          "Velocity", "NodeMass"]


def solo(p, n):
    from mahyco_b200 import Hydro
    with Hydro(p) as h:
        h.hydroStartInit()
        h.cycle(n)
        assert h.synchronize() == 0
        return {f: h.field(f) for f in FIELDS}, h.scalars()


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [False, True], ids=["launches", "graph"])
def test_batch_matches_solo(graph):
    from mahyco_b200 import Batch
    names = sorted(PARITY_CASES)
    params = [PARITY_CASES[n][0]() for n in names]
    params += [seeded_two_state(s, n) for s, n in ((1, 17), (2, 40), (3, 23))]
    ncycles = 24
    with Batch() as b:
        idx = [b.add(p) for p in params]
        b.init()
        b.cycle(ncycles, graph=graph)
        b.synchronize()
        for i, p in zip(idx, params):
            ref, s_ref = solo(p, ncycles)
            s = b.scalars(i)
            assert s["status"] == 0 and s["iteration"] == ncycles
            assert s["time"] == s_ref["time"] and s["deltat"] == s_ref["deltat"]
            for f in FIELDS:
                assert np.array_equal(b.field(i, f), ref[f]), (i, f)


@pytest.mark.gpu
def test_failing_case_leaves_neighbours_intact():
    """A case forced into a time-step underflow (deltat-min above every
    admissible step: injected from the host) retires itself; the other cases
    of the batch keep running and match their solo runs."""
    from mahyco_b200 import Batch, ST_DT_UNDERFLOW
    good = [seeded_two_state(s, 24) for s in (5, 6)]
    bad = seeded_two_state(7, 24)
    bad.deltat_min = 1.0
    with Batch() as b:
        ig = [b.add(p) for p in good]
        ib = b.add(bad)
        b.init()
        b.cycle(12)
        b.synchronize()
        sb = b.scalars(ib)
        assert sb["status"] & ST_DT_UNDERFLOW and sb["iteration"] <= 1
        for i, p in zip(ig, good):
            ref, _ = solo(p, 12)
            assert b.scalars(i)["status"] == 0
            for f in FIELDS:
                assert np.array_equal(b.field(i, f), ref[f])


@pytest.mark.gpu
def test_iteration_limits_and_removal():
    from mahyco_b200 import Batch
    ps = [seeded_two_state(s, 20) for s in (11, 12, 13)]
    with Batch() as b:
        i0 = b.add(ps[0], iteration_limit=5)
        i1 = b.add(ps[1])
        b.init()
        b.cycle(8)
        assert b.scalars(i0)["iteration"] == 5
        assert b.scalars(i1)["iteration"] == 8
        ref0, _ = solo(ps[0], 5)
        assert np.array_equal(b.field(i0, "Density"), ref0["Density"])
        b.remove(i0)
        i2 = b.add(ps[2])      # joins mid-flight with its own sweep rotation
        b.init()
        b.cycle(7)
        b.synchronize()
        ref1, _ = solo(ps[1], 15)
        ref2, _ = solo(ps[2], 7)
        assert np.array_equal(b.field(i1, "Density"), ref1["Density"])
        assert np.array_equal(b.field(i2, "Density"), ref2["Density"])
