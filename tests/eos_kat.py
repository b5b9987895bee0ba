"""Known answers of the three equation-of-state services, written from
their formulas (PerfectGasEOSService.cc:45-67, StiffenedGasEOSService.cc:
43-63, MieGruneisenEOSService.cc:44-97; initEOS: PG 12-35, SG 14-33, MG
12-34):

* ``*_float`` evaluate the formula in double precision in the services'
  operation order, so IEEE arithmetic gives the exact bits an implementation
  in that order must produce (perfect and stiffened gas);
* ``mg_exact`` evaluates the Mie-Gruneisen pressure in exact rational
  arithmetic on the double inputs, against which an implementation is held
  to a stated relative bound (its result rounds several times).
"""
import math
from fractions import Fraction

# states (rho, e) per law, spanning compression and expansion
PG_STATES = [(1.0, 2.5), (0.125, 2.0), (3.7, 0.01), (1e-3, 1e5)]
SG_STATES = [(1000.0, 1.0e6), (1020.0, 8.3e5), (990.0, 2.1e6)]
MG_STATES = [(2800.0, 1.0e6), (2710.0, 0.0), (2650.0, 5.0e5), (3100.0, 2.0e7)]


def pg_float(gamma, rho, e):
    p = (gamma - 1.) * rho * e
    c = math.sqrt(gamma * p / rho)
    return p, c, (gamma - 1.) * rho


def sg_float(gamma, pinf, rho, e):
    p = ((gamma - 1.) * rho * e) - (gamma * pinf)
    c = math.sqrt((gamma / rho) * (p + pinf))
    return p, c, (gamma - 1.) * rho


def pg_init_float(gamma, p, rho):
    return p / ((gamma - 1.) * rho), math.sqrt(gamma * p / rho)


def sg_init_float(gamma, pinf, p, rho):
    return (p + (gamma * pinf)) / ((gamma - 1.) * rho), math.sqrt((gamma / rho) * (p + pinf))


def mg_exact(o, rho, e):
    """Exact pressure and dp/de of the Mie-Gruneisen law (the reference uses
    s2 in both the mu^2 and mu^3 terms of the denominator)."""
    F = Fraction
    rho0, c0, s1, s2, g0, a = (F(x) for x in (o.rho0, o.c0, o.s1, o.s2, o.gamma0, o.a))
    J = rho0 / F(rho)
    mu = 1 / J - 1
    if mu > 0:
        num = rho0 * c0 ** 2 * mu * (1 + (1 - g0 / 2) * mu - a * mu ** 2 / 2)
        den = (1 - (s1 - 1) * mu - s2 * mu ** 2 / (1 + mu) - s2 * mu ** 3 / (1 + mu) ** 2) ** 2
        p = num / den + (g0 + a * mu) * F(e)
    else:
        p = rho0 * c0 ** 2 * mu + (g0 + a * mu) * F(e)
    return p, g0 + a * mu


def mg_sound_exact(o, rho, e):
    """sqrt((p(rho + 1e-7) - p(rho - 1e-7)) / 2e-7), the services' finite
    difference (1e4 when not positive), from exact pressures at the two
    rounded densities."""
    p1, _ = mg_exact(o, rho - 1.e-7, e)
    p2, _ = mg_exact(o, rho + 1.e-7, e)
    d = p2 - p1
    return math.sqrt(float(d / Fraction(2.e-7))) if d > 0 else 1.e4


def rel(a, b):
    b = float(b)
    return abs(a - b) / abs(b) if b != 0 else abs(a)
