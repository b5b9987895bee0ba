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
