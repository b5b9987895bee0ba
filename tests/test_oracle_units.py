"""Known-answer tests of the oracle's building blocks, derived from the
formulas of the reference (no golden pins these paths)."""
import math
import random
from decimal import Decimal, getcontext

import pytest

from mahyco_b200.case import EnvParams, env_defaults, EOS_PERFECT_GAS, EOS_STIFFENED_GAS
from tests.oracle import eos_point, lib, setup_kat


def test_limiters_known_values():
    # UtilesRemap.cc:108-120
    L = setup_kat(lib())
    table = {  # r: (minmod, superbee, vanleer)
        -1.0: (0.0, 0.0, 0.0), 0.0: (0.0, 0.0, 0.0), 0.5: (0.5, 1.0, 2 * 0.5 / 1.5),
        1.0: (1.0, 1.0, 1.0), 2.0: (1.0, 2.0, 4.0 / 3.0), 3.0: (1.0, 2.0, 1.5)}
    for r, vals in table.items():
        for lid, v in enumerate(vals):
            assert L.oracle_flux_limiter(lid, r) == v, (lid, r)


def test_limited_gradient_symmetric_and_monotone():
    L = setup_kat(lib())
    for lid in range(3):
        assert L.oracle_limited_gradient(lid, 2.0, 2.0) == 2.0
        assert L.oracle_limited_gradient(lid, -1.0, 1.0) == 0.0
        assert L.oracle_limited_gradient(lid, 0.0, 3.0) == 0.0


def test_stiffened_gas_reduces_to_perfect_gas():
    pg, sg = EnvParams(), EnvParams()
    env_defaults(pg, EOS_PERFECT_GAS)
    env_defaults(sg, EOS_STIFFENED_GAS)
    sg.limit_tension = 0.0
    for rho, e in ((1.0, 2.5), (0.125, 2.0), (1000.0, 1e6)):
        assert eos_point(pg, rho, e) == eos_point(sg, rho, e)


def test_stiffened_gas_formula():
    sg = EnvParams()
    env_defaults(sg, EOS_STIFFENED_GAS)
    sg.adiabatic_cst, sg.limit_tension = 4.4, 6e8
    p, c = eos_point(sg, 1000.0, 1.0e6)
    assert p == ((4.4 - 1.) * 1000.0 * 1.0e6) - (4.4 * 6e8)
    assert c == math.sqrt((4.4 / 1000.0) * (p + 6e8))


def test_cube_root_power_correctly_rounded():
    getcontext().prec = 60
    L = lib()
    y = Decimal(1.0 / 3.0)
    rng = random.Random(7)
    for _ in range(3000):
        x = rng.uniform(1e-10, 10.0) if rng.random() < 0.5 else 10 ** rng.uniform(-12, 3)
        r = L.oracle_pow_third_cr(x)
        exact = Decimal(x) ** y
        assert abs(Decimal(r) - exact) <= Decimal(math.ulp(r)) / 2, x


def test_five_thirds_power_correctly_rounded():
    """NewHypoModel's J^(5./3.) (the double nearest to 5/3 as exponent)."""
    getcontext().prec = 60
    L = lib()
    y = Decimal(5.0 / 3.0)
    rng = random.Random(11)
    for _ in range(3000):
        x = rng.uniform(0.5, 2.0) if rng.random() < 0.5 else 10 ** rng.uniform(-6, 6)
        r = L.oracle_pow_five_thirds_cr(x)
        exact = Decimal(x) ** y
        assert abs(Decimal(r) - exact) <= Decimal(math.ulp(r)) / 2, x


def test_cube_correctly_rounded():
    getcontext().prec = 60
    L = lib()
    rng = random.Random(3)
    for _ in range(3000):
        x = rng.uniform(-1.0, 1.0)
        r = L.oracle_cube_cr(x)
        exact = Decimal(x) ** 3
        assert abs(Decimal(r) - exact) <= Decimal(math.ulp(r)) / 2, x


def test_glibc_pow_is_not_correctly_rounded():
    """Why the parity tests run a correctly rounded oracle: the reference's
    std::pow(V, 0.5) differs from the correctly rounded sqrt(V) for a small
    fraction of inputs."""
    import ctypes
    libm = ctypes.CDLL("libm.so.6")
    libm.pow.restype = ctypes.c_double
    libm.pow.argtypes = [ctypes.c_double, ctypes.c_double]
    rng = random.Random(11)
    diff = sum(libm.pow(x, 0.5) != math.sqrt(x) for x in (rng.uniform(1e-4, 1e-2) for _ in range(200000)))
    assert 0 < diff < 2000


# --- known answers of the three equations of state (tests/eos_kat.py) ------
from mahyco_b200.case import EOS_MIE_GRUNEISEN  # noqa: E402
from tests import eos_kat  # noqa: E402


def _env(eos, **kw):
    o = EnvParams()
    env_defaults(o, eos)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def test_perfect_gas_known_answers():
    o = _env(EOS_PERFECT_GAS, adiabatic_cst=1.4)
    for rho, e in eos_kat.PG_STATES:
        assert eos_point(o, rho, e, with_dpde=True) == eos_kat.pg_float(1.4, rho, e), (rho, e)
    # by hand: gamma 5/3, rho 3, e 0.5 -> p = (2/3) 3 0.5 = 1, c^2 = 5/9
    o = _env(EOS_PERFECT_GAS, adiabatic_cst=5.0 / 3.0)
    p, c, d = eos_point(o, 3.0, 0.5, with_dpde=True)
    assert abs(p - 1.0) <= 2e-16 and abs(c - math.sqrt(5.0 / 9.0)) <= 2e-16 and abs(d - 2.0) <= 4e-16


def test_stiffened_gas_known_answers():
    o = _env(EOS_STIFFENED_GAS, adiabatic_cst=4.4, limit_tension=6e8)
    for rho, e in eos_kat.SG_STATES:
        assert eos_point(o, rho, e, with_dpde=True) == eos_kat.sg_float(4.4, 6e8, rho, e), (rho, e)
    # by hand: gamma 2, p_inf 1, rho 1, e 3 -> p = 3 - 2 = 1, c = sqrt(2 (1 + 1)) = 2, dp/de = 1
    o = _env(EOS_STIFFENED_GAS, adiabatic_cst=2.0, limit_tension=1.0)
    assert eos_point(o, 1.0, 3.0, with_dpde=True) == (1.0, 2.0, 1.0)


def test_stiffened_gas_at_zero_p_inf_is_perfect_gas():
    for g in (1.4, 5.0 / 3.0, 4.4):
        pg = _env(EOS_PERFECT_GAS, adiabatic_cst=g)
        sg = _env(EOS_STIFFENED_GAS, adiabatic_cst=g, limit_tension=0.0)
        for rho, e in eos_kat.PG_STATES:
            a, b = eos_point(pg, rho, e, with_dpde=True), eos_point(sg, rho, e, with_dpde=True)
            assert a[0] == b[0] and a[2] == b[2]
            # sqrt(g p / rho) against sqrt((g / rho) p): one rounding apart
            assert abs(a[1] - b[1]) <= 2 * math.ulp(a[1])


def test_mie_gruneisen_known_answers():
    o = _env(EOS_MIE_GRUNEISEN, rho0=2710.0, c0=5328.0, s1=1.338, gamma0=2.0)
    for rho, e in eos_kat.MG_STATES:
        p, c, d = eos_point(o, rho, e, with_dpde=True)
        pe, de = eos_kat.mg_exact(o, rho, e)
        assert eos_kat.rel(p, pe) <= 1e-13 or abs(p - float(pe)) <= 1e-13 * 1e9, (rho, e, p, float(pe))
        assert eos_kat.rel(d, de) <= 1e-15, (rho, e)
        # the sound speed is a finite difference of two pressures of ~3e9
        # that differ by ~6: a few tens of ulps (4.8e-7 each) of rounding in
        # each pressure make up to ~5e-6 of p2 - p1, ~2.5e-6 of c
        assert eos_kat.rel(c, eos_kat.mg_sound_exact(o, rho, e)) <= 5e-6, (rho, e)
    # by hand, at the reference density: mu = 0, p = Gamma0 e, dp/de = Gamma0
    p, c, d = eos_point(o, 2710.0, 123.0, with_dpde=True)
    assert (p, d) == (2.0 * 123.0, 2.0)


def test_sedov_box_corner_reach():
    """Two oracle Sedov boxes of the same cell size (16^3 and 32^3 on the
    origin corner; power-of-two sides keep the cell width bitwise equal)
    agree on the corner [0, 16 - (3 + 2N))^3 after N cycles: the far walls
    reach no deeper than the margin that the 384^3 corner comparison of
    tests/test_gpu_fullsize.py leaves out."""
    import numpy as np
    from mahyco_b200.cases import workload
    from tests.oracle import Oracle
    from tests.test_gpu_fullsize import sedov_corner_margin
    A, B, N = 16, 32, 5
    k = A - sedov_corner_margin(N)
    oa, ob = Oracle(workload("sedov3d", scale=A / 384), cr_pow=True), Oracle(workload("sedov3d", scale=B / 384), cr_pow=True)
    assert oa.init() == 0 and ob.init() == 0 and oa.iterate(N) == 0 and ob.iterate(N) == 0
    assert oa.scalar("deltat") == ob.scalar("deltat")
    for f in ("Density", "InternalEnergy", "Pressure", "CellMass"):
        assert np.array_equal(oa.field(f).reshape(A, A, A)[:k, :k, :k], ob.field(f).reshape(B, B, B)[:k, :k, :k]), f
    va = oa.field("Velocity").reshape(A + 1, A + 1, A + 1, 3)[:k, :k, :k]
    vb = ob.field("Velocity").reshape(B + 1, B + 1, B + 1, 3)[:k, :k, :k]
    assert np.array_equal(va, vb)
