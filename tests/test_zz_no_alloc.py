"""The allocation-free CFL time step (mhc_cfl_delta_t_noalloc) against the
case entry point mhc_compute_delta_t.

The allocation-free variant exists for callers that cannot allocate device
memory themselves at the point where they need a time step -- codes that
hand all device memory out through their own pool or run where allocation
is not permitted -- so it takes the caller's device buffers and keeps its
reduction scratch in a fixed array inside the library.  This file is
collected last on purpose (tests/test_zz_*), and it must pass both alone in
a fresh process and after the rest of the suite, because the scratch array
persists between calls.
"""
import ctypes

import numpy as np
import pytest


@pytest.mark.gpu
def test_noalloc_cfl_matches_case_entry_point_twice():
    import torch
    import mahyco_b200 as mb
    from mahyco_b200.cases import sod, SUPERBEE
    lib = mb.load()
    p = sod(dim=3, n=(64, 16, 16), L=(1.0, 0.25, 0.25), bi=True, limiter=SUPERBEE, deltat_init=1e-3)
    with mb.Hydro(p, lib) as h:
        h.hydroStartInit()
        h.cycle(9)
        assert h.synchronize() == 0
        dt_prev = h.scalars()["deltat"]
        out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        for call in range(2):  # two calls in a row share the scratch array
            h.cycle(1)  # the case's own computeDeltaT (mhc_compute_delta_t)
            assert h.synchronize() == 0
            expect = h.scalars()["deltat"]
            l = torch.from_numpy(h.field("CaracteristicLength")).cuda()
            c = torch.from_numpy(h.field("SoundSpeed")).cuda()
            v = h.field("Velocity").reshape(-1, 3)
            vx, vy, vz = (torch.from_numpy(np.ascontiguousarray(v[:, q])).cuda() for q in range(3))
            torch.cuda.synchronize()
            stream = torch.cuda.current_stream().cuda_stream
            rc = lib.mhc_cfl_delta_t_noalloc(p.dim, p.nx, p.ny, p.nz, l.data_ptr(), c.data_ptr(),
                                             vx.data_ptr(), vy.data_ptr(), vz.data_ptr(), p.cfl, dt_prev,
                                             p.deltat_max, p.deltat_min, out.data_ptr(), stream)
            assert rc == 0, lib.mhc_noalloc_last_error()
            torch.cuda.synchronize()
            got = out.item()
            assert got == expect, (call, got, expect)
            dt_prev = expect


@pytest.mark.gpu
def test_noalloc_rejects_meshes_above_its_scratch():
    import torch
    import mahyco_b200 as mb
    lib = mb.load()
    t = torch.zeros(4, dtype=torch.float64, device="cuda")
    n = 256  # 256^3 cells > MHC_NOALLOC_MAX_CELLS
    rc = lib.mhc_cfl_delta_t_noalloc(3, n, n, n, t.data_ptr(), t.data_ptr(), t.data_ptr(), t.data_ptr(),
                                     t.data_ptr(), 0.3, 1.0, 1.0, 0.0, t.data_ptr(), None)
    assert rc == -1
    assert b"at most" in lib.mhc_noalloc_last_error()
