"""The measured workloads at their full sizes (mahyco_b200.cases.workload).

* 3D BiSod 256x64x64, 2 materials, superbee (the headline bench line): 10
  cycles on the GPU and in the oracle with correctly rounded powers; every
  cell, environment and node field and the time-loop scalars must be
  bit-identical, as on the small parity cases.
* 3D Sedov 384^3 (56.6 M cells, 22 GB on the device; the sequential oracle
  would need about 60 GB of host memory): size-independent properties.  Two
  runs of the same case give bit-identical fields (no atomics in any sum:
  every reduction has a fixed order), and the remap moves mass between
  cells only, so the total mass is conserved to rounding.
* 3D Sedov 384^3 against the oracle on its origin corner: a 64^3 box of
  the same cell size (L = 1.2 * 64 / 384 gives bitwise the same cell width,
  64 being a power of two), the same energy, background pressure and first
  time step.  The box's far walls (free boundaries where the full mesh has
  neighbours) change the box's fields from there inwards by at most
  2 + N cells after N cycles (measured with two oracle boxes,
  tests/test_oracle_units.py::test_sedov_box_corner_reach), so the corner
  [0, 64 - (3 + 2N))^3 of the GPU's full mesh must equal the oracle box
  bit for bit, as must the time step and time.
"""
import numpy as np
import pytest

from mahyco_b200.cases import workload
from tests.test_gpu_parity import compare


@pytest.mark.gpu
def test_bisod_256x64x64_bit_identical_to_oracle():
    from mahyco_b200 import Hydro
    from tests.oracle import Oracle
    p = workload("bisod3d")
    n = 10
    ora = Oracle(p, cr_pow=True)
    assert ora.init() == 0
    gpu = Hydro(p)
    gpu.hydroStartInit()
    assert max(compare(gpu, ora, p.nb_env).values()) == 0.0
    gpu.cycle(n)
    assert gpu.synchronize() == 0
    assert ora.iterate(n) == 0
    errs = compare(gpu, ora, p.nb_env)
    s = gpu.scalars()
    errs["time"] = abs(s["time"] - ora.scalar("time"))
    errs["deltat"] = abs(s["deltat"] - ora.scalar("deltat"))
    gpu.close()
    bad = {k: v for k, v in errs.items() if v != 0.0}
    assert not bad, bad


def _sedov_run(n):
    from mahyco_b200 import Hydro
    p = workload("sedov3d")
    h = Hydro(p)
    h.hydroStartInit()
    m0 = h.field("CellMass")
    h.cycle(n)
    st = h.synchronize()
    out = {f: h.field(f) for f in ("Density", "Pressure", "InternalEnergy", "CellMass")}
    out["Velocity"] = h.field("Velocity")
    s = h.scalars()
    h.close()
    return st, m0, out, s


@pytest.mark.gpu
def test_sedov_384_cubed_deterministic_and_mass_conserving():
    n = 4
    st1, m0, a, s1 = _sedov_run(n)
    assert st1 == 0 and s1["iteration"] == n
    assert all(np.isfinite(v).all() for v in a.values())
    st2, _, b, s2 = _sedov_run(n)
    assert st2 == 0 and (s1["time"], s1["deltat"]) == (s2["time"], s2["deltat"])
    for f in a:
        assert np.array_equal(a[f], b[f]), f
    total0, total = m0.sum(dtype=np.float64), a["CellMass"].sum(dtype=np.float64)
    assert abs(total - total0) <= 1e-12 * abs(total0), (total0, total)
    # the blast has moved: the origin cell expanded and its energy reached
    # neighbours (the background energy is p0 / ((gamma - 1) rho) = 2.5e-6)
    assert a["Density"][0] < 1.0 and (a["InternalEnergy"] > 1e-3).sum() > 1


SEDOV_BOX, SEDOV_BOX_CYCLES = 64, 16


def sedov_corner_margin(ncycles: int) -> int:
    """Cells next to the box walls left out of the comparison after
    ncycles: twice the measured reach of the walls (2 + N cells)."""
    return 3 + 2 * ncycles


@pytest.mark.gpu
def test_sedov_384_cubed_origin_corner_matches_oracle_box():
    from mahyco_b200 import Hydro
    from tests.oracle import Oracle
    B, N = SEDOV_BOX, SEDOV_BOX_CYCLES
    k = B - sedov_corner_margin(N)
    full, box = workload("sedov3d"), workload("sedov3d", scale=B / 384)
    assert box.nx == B and box.lx / box.nx == full.lx / full.nx and box.deltat_init == full.deltat_init
    ora = Oracle(box, cr_pow=True)
    assert ora.init() == 0 and ora.iterate(N) == 0
    h = Hydro(full)
    h.hydroStartInit()
    h.cycle(N)
    assert h.synchronize() == 0
    s = h.scalars()
    assert s["iteration"] == N
    assert (s["time"], s["deltat"]) == (ora.scalar("time"), ora.scalar("deltat"))
    n = full.nx
    for f in ("Density", "InternalEnergy", "Pressure", "SoundSpeed", "CellMass", "PseudoViscosity"):
        g = h.field(f).reshape(n, n, n)[:k, :k, :k]
        o = ora.field(f).reshape(B, B, B)[:k, :k, :k]
        assert np.array_equal(g, o), f
    g = h.field("Velocity").reshape(n + 1, n + 1, n + 1, 3)[:k, :k, :k]
    o = ora.field("Velocity").reshape(B + 1, B + 1, B + 1, 3)[:k, :k, :k]
    assert np.array_equal(g, o)
    # the blast has left the origin cell within the compared corner
    e = h.field("InternalEnergy").reshape(n, n, n)
    assert (e[:k, :k, :k] > 1e-3).sum() > 1
    h.close()
