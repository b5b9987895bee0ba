"""Test-side binding of the CPU oracle (oracle/liboracle_mahyco.so).

The oracle restates the reference cycle on the CPU; it is only a checker for
the CUDA library.  It is built by ``make -C oracle`` (also run by
``__graft_entry__.build()``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from mahyco_b200.case import CaseParams

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle_mahyco.so")
_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(ORACLE_LIB):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    L = C.CDLL(ORACLE_LIB)
    L.oracle_create.restype = C.c_void_p
    L.oracle_create.argtypes = [C.POINTER(CaseParams)]
    L.oracle_destroy.argtypes = [C.c_void_p]
    L.oracle_init.argtypes = [C.c_void_p]
    L.oracle_iterate.argtypes = [C.c_void_p, C.c_int]
    L.oracle_run.argtypes = [C.c_void_p, C.c_long]
    L.oracle_scalar.restype = C.c_double
    L.oracle_scalar.argtypes = [C.c_void_p, C.c_char_p]
    L.oracle_get_field.restype = C.c_long
    L.oracle_get_field.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.POINTER(C.c_double), C.c_long]
    L.oracle_eos_apply.argtypes = [C.c_void_p, C.c_int]
    L.oracle_set_initial_field.restype = C.c_int
    L.oracle_set_initial_field.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.c_long]
    L.oracle_set_field.restype = C.c_long
    L.oracle_set_field.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.POINTER(C.c_double), C.c_long]
    L.oracle_th_count.restype = C.c_long
    L.oracle_th_count.argtypes = [C.c_void_p]
    L.oracle_th_line.argtypes = [C.c_void_p, C.c_long, C.POINTER(C.c_double)]
    L.oracle_set_option.argtypes = [C.c_void_p, C.c_char_p, C.c_double]
    L.oracle_pow_third_cr.restype = C.c_double
    L.oracle_pow_third_cr.argtypes = [C.c_double]
    L.oracle_cube_cr.restype = C.c_double
    L.oracle_cube_cr.argtypes = [C.c_double]
    L.oracle_pow_five_thirds_cr.restype = C.c_double
    L.oracle_pow_five_thirds_cr.argtypes = [C.c_double]
    _lib = L
    return L


class Oracle:
    """cr_pow=False follows the reference literally (std::pow of glibc);
    cr_pow=True evaluates the same powers correctly rounded, as the CUDA
    library does."""

    def __init__(self, params: CaseParams, cr_pow: bool = False):
        self.L = lib()
        self.params = params
        self.h = self.L.oracle_create(C.byref(params))
        self.ncell, self.nnode = params.ncell, params.nnode
        self.set_option("cr_pow", 1.0 if cr_pow else 0.0)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_destroy(self.h)
            self.h = None

    def set_option(self, name: str, value: float):
        assert self.L.oracle_set_option(self.h, name.encode(), float(value)) == 0

    def init(self) -> int:
        return self.L.oracle_init(self.h)

    def iterate(self, n: int) -> int:
        return self.L.oracle_iterate(self.h, n)

    def run(self, max_iter: int = 10**9) -> int:
        return self.L.oracle_run(self.h, max_iter)

    def scalar(self, name: str) -> float:
        return self.L.oracle_scalar(self.h, name.encode())

    def field(self, name: str, env: int = -1) -> np.ndarray:
        n = 3 * (self.ncell if name == "CellCoord" else self.nnode) if name in ("Velocity", "VelocityN", "NodeCoord", "CellCoord") else (
            self.nnode if name == "NodeMass" else self.ncell)
        out = np.empty(n, dtype=np.float64)
        got = self.L.oracle_get_field(self.h, name.encode(), env, out.ctypes.data_as(C.POINTER(C.c_double)), n)
        assert got == n, (name, got)
        return out

    def set_initial_field(self, name: str, values) -> None:
        """EXTERNAL initial state / mesh-file node coordinates, before init()."""
        a = np.ascontiguousarray(values, dtype=np.float64)
        got = self.L.oracle_set_initial_field(self.h, name.encode(), a.ctypes.data_as(C.POINTER(C.c_double)), a.size)
        assert got > 0, (name, got)

    def set_field(self, name: str, values: np.ndarray, env: int = -1) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64)
        got = self.L.oracle_set_field(self.h, name.encode(), env, a.ctypes.data_as(C.POINTER(C.c_double)), a.size)
        assert got > 0, (name, got)

    def eos_apply(self, env: int) -> None:
        assert self.L.oracle_eos_apply(self.h, env) == 0

    def time_history(self) -> np.ndarray:
        n = self.L.oracle_th_count(self.h)
        w = 1 + 5 * self.params.nb_env
        buf = (C.c_double * w)()
        rows = []
        for i in range(n):
            self.L.oracle_th_line(self.h, i, buf)
            rows.append(list(buf))
        return np.array(rows).reshape(-1, w)


def setup_kat(L):
    L.oracle_flux_limiter.restype = C.c_double
    L.oracle_flux_limiter.argtypes = [C.c_int, C.c_double]
    L.oracle_limited_gradient.restype = C.c_double
    L.oracle_limited_gradient.argtypes = [C.c_int, C.c_double, C.c_double]
    from mahyco_b200.case import EnvParams
    L.oracle_eos_point.argtypes = [C.POINTER(EnvParams), C.c_double, C.c_double,
                                   C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    return L


def eos_point(env, rho, e, with_dpde=False):
    """(p, c) of the oracle's applyEOS at one state; (p, c, dp/de) with
    with_dpde."""
    L = setup_kat(lib())
    p, c, d = C.c_double(), C.c_double(), C.c_double()
    L.oracle_eos_point(C.byref(env), rho, e, C.byref(p), C.byref(c), C.byref(d))
    return (p.value, c.value, d.value) if with_dpde else (p.value, c.value)
