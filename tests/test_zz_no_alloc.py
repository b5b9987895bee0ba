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
import numpy as np
import pytest


def _check_two_calls(p, warm_cycles, euler_full, expect_check=None):
    """Runs a case, then twice in a row: one iteration of the case (its own
    computeDeltaT), and the allocation-free entry point on the same state
    with the previous deltat; both must give the same deltat exactly."""
    import torch
    import mahyco_b200 as mb
    lib = mb.load()
    with mb.Hydro(p, lib) as h:
        h.hydroStartInit()
        h.cycle(warm_cycles)
        assert h.synchronize() == 0
        dt_prev = h.scalars()["deltat"]
        out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        for call in range(2):  # two calls in a row share the scratch array
            h.cycle(1)  # the case's own computeDeltaT (mhc_compute_delta_t)
            assert h.synchronize() == 0
            expect = h.scalars()["deltat"]
            if expect_check is not None:
                expect_check(expect, dt_prev)
            l = torch.from_numpy(h.field("CaracteristicLength")).cuda()
            c = torch.from_numpy(h.field("SoundSpeed")).cuda()
            v = h.field("Velocity").reshape(-1, 3)
            vx, vy, vz = (torch.from_numpy(np.ascontiguousarray(v[:, q])).cuda() for q in range(3))
            torch.cuda.synchronize()
            stream = torch.cuda.current_stream().cuda_stream
            ptrs = (vx.data_ptr(), vy.data_ptr(), vz.data_ptr()) if euler_full else (None, None, None)
            rc = lib.mhc_cfl_delta_t_noalloc(p.dim, p.nx, p.ny, p.nz, l.data_ptr(), c.data_ptr(), *ptrs,
                                             1 if euler_full else 0, p.cfl, dt_prev, p.deltat_max,
                                             p.deltat_min, out.data_ptr(), stream)
            assert rc == 0, lib.mhc_noalloc_last_error()
            torch.cuda.synchronize()
            got = out.item()
            assert got == expect, (call, got, expect)
            dt_prev = expect


@pytest.mark.gpu
def test_noalloc_cfl_matches_case_entry_point_twice():
    """3D two-material ADI remap, is-euler-scheme Full: node speeds count."""
    from mahyco_b200.cases import sod, SUPERBEE
    p = sod(dim=3, n=(64, 16, 16), L=(1.0, 0.25, 0.25), bi=True, limiter=SUPERBEE, deltat_init=1e-3)
    _check_two_calls(p, 9, euler_full=True)


@pytest.mark.gpu
def test_noalloc_cfl_2d_per_axis_euler_leaves_node_speed_out():
    """2D Sedov with is-euler-scheme X: computeDeltaT drops the node speed,
    and so does the allocation-free variant with euler_full = 0."""
    from mahyco_b200.cases import sedov, EULER_X
    p = sedov(dim=2, n=(24, 24), deltat_init=1e-4)
    p.is_euler_scheme = EULER_X
    _check_two_calls(p, 20, euler_full=False)


@pytest.mark.gpu
def test_noalloc_cfl_2d_lagrange_with_deltat_max_bound_active():
    """2D Lagrangian Sod whose deltat_max bound decides the step."""
    from mahyco_b200.cases import sod
    p = sod(dim=2, n=(60, 5), L=(1.0, 0.1), bi=False, remap=False, deltat_max=2e-5, deltat_init=2e-5)

    def bound_active(dt, dt_prev):
        assert dt == p.deltat_max, dt

    _check_two_calls(p, 10, euler_full=True, expect_check=bound_active)


@pytest.mark.gpu
def test_noalloc_rejects_meshes_above_its_scratch():
    import torch
    import mahyco_b200 as mb
    lib = mb.load()
    t = torch.zeros(4, dtype=torch.float64, device="cuda")
    n = 256  # 256^3 cells > MHC_NOALLOC_MAX_CELLS
    rc = lib.mhc_cfl_delta_t_noalloc(3, n, n, n, t.data_ptr(), t.data_ptr(), t.data_ptr(), t.data_ptr(),
                                     t.data_ptr(), 1, 0.3, 1.0, 1.0, 0.0, t.data_ptr(), None)
    assert rc == -1
    assert b"at most" in lib.mhc_noalloc_last_error()
