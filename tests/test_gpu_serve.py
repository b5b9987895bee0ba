"""Serving: continuous batching under an HBM budget (mhc_server_*).

Requests join while others are on the GPU; each result must be the same
alone and in the mix (bitwise: batching never changes a case's arithmetic),
the budget must hold at every step, and the per-request failure statuses
(admission, timeout) must be reported without disturbing the other cases.
"""
import numpy as np
import pytest

import mahyco_b200 as mb
from mahyco_b200.cases import serving_request, bar_impact

pytestmark = pytest.mark.gpu

FIELDS = ("Density", "Pressure", "InternalEnergy", "Velocity")

MIX = [("sedov2d", 900, 30), ("bisod3d", 2000, 25), ("water_bubbles", 1000, 40), ("sedov3d", 1000, 20),
       ("bar", 0, 30), ("sedov2d", 3000, 15), ("bisod3d", 500, 35), ("water_bubbles", 250, 20)]


def _params(kind, cells):
    return bar_impact(n=(8, 40)) if kind == "bar" else serving_request(kind, cells)


def _alone(p, iterations):
    h = mb.Hydro(p)
    h.hydroStartInit()
    h.cycle(iterations)
    out = {f: h.field(f) for f in FIELDS}
    sc = h.scalars()
    h.close()
    return out, sc


def test_served_results_equal_alone():
    srv = mb.Server()
    tickets = []
    # arrivals spread over the run: two requests join before every step
    pending = list(MIX)
    while pending or srv.stats()["running"] or srv.stats()["queued"]:
        for _ in range(2):
            if pending:
                kind, cells, its = pending.pop(0)
                tickets.append((srv.submit(_params(kind, cells), its), kind, cells, its))
        srv.step(3)
    for t, kind, cells, its in tickets:
        st = srv.poll(t)
        assert st["state"] == mb.REQ_DONE, (kind, st)
        assert st["iteration"] == its
        ref, sc = _alone(_params(kind, cells), its)
        for f in FIELDS:
            np.testing.assert_array_equal(srv.fetch(t, f), ref[f], err_msg=f"{kind} {f}")
        assert st["time"] == sc["time"]
        tm = srv.times(t)
        assert tm["submit"] <= tm["admit"] <= tm["done"]
        srv.release(t)
    assert srv.stats()["bytes_in_use"] == 0
    srv.close()


def test_budget_admission_and_backfill():
    lib = mb.load()
    reqs = [_params(k, c) for k, c, _ in MIX]
    import ctypes as C
    lib.mhc_case_device_bytes.restype = C.c_longlong
    sizes = [lib.mhc_case_device_bytes(C.byref(p)) for p in reqs]
    budget = max(sizes) + min(sizes)  # the biggest case plus the smallest fits, never two big ones
    srv = mb.Server(hbm_budget_bytes=budget)
    tickets = [srv.submit(p, 10) for p in reqs]
    peak = 0
    for _ in range(500):
        srv.step(2)
        s = srv.stats()
        peak = max(peak, s["bytes_in_use"])
        assert s["bytes_in_use"] <= budget
        for t in tickets:
            if t in srv.params and srv.poll(t)["state"] == mb.REQ_DONE:
                srv.release(t)
        if not s["queued"] and not s["running"]:
            break
    assert peak > 0
    for t in tickets:
        assert t not in srv.params  # every request ran to completion and was released
    srv.close()


def test_oversize_request_refused_and_timeout():
    import ctypes as C
    lib = mb.load()
    lib.mhc_case_device_bytes.restype = C.c_longlong
    small = _params("sedov2d", 400)
    big = _params("sedov3d", 30000)
    srv = mb.Server(hbm_budget_bytes=lib.mhc_case_device_bytes(C.byref(small)) * 2)
    t_big = srv.submit(big, 5)
    t_ok = srv.submit(small, 5)
    t_late = srv.submit(_params("sedov2d", 400), 10 ** 9, timeout_s=0.05)
    for _ in range(200):
        srv.step(5)
        if srv.poll(t_late)["state"] == mb.REQ_FAILED and srv.poll(t_ok)["state"] == mb.REQ_DONE:
            break
    b = srv.poll(t_big)
    assert b["state"] == mb.REQ_FAILED and b["status"] & mb.ST_OOM_ADMISSION
    assert srv.poll(t_ok)["state"] == mb.REQ_DONE
    late = srv.poll(t_late)
    assert late["state"] == mb.REQ_FAILED and late["status"] & mb.ST_TIMEOUT
    with pytest.raises(mb.MahycoError):
        srv.release(999999)
    srv.release(t_ok)
    srv.release(t_late)
    srv.release(t_big)
    srv.close()
