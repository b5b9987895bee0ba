"""The C ABI library loads without a GPU, exports every symbol that
include/*.h declares, and fails loudly (an error code, no CPU fallback) when
no CUDA device is available."""
import ctypes
import os
import re

import pytest

import mahyco_b200 as mb

HERE = os.path.dirname(os.path.abspath(__file__))
INCLUDE = os.path.join(os.path.dirname(HERE), "include")


def declared_symbols():
    names = set()
    for h in os.listdir(INCLUDE):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(mhc_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = mb.load()
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert declared_symbols() <= set(mb._SIGS)


def test_version_and_budget_query():
    lib = mb.load()
    assert b"sm_100a" in lib.mhc_version()
    p = mb.default_params()
    p.dim, p.nx, p.ny, p.nz, p.nb_env = 3, 64, 64, 64, 2
    assert lib.mhc_case_device_bytes(ctypes.byref(p)) > 64 ** 3 * 8 * 20


def test_rejects_options_outside_the_hot_path():
    """Options outside the implemented path are refused before any device
    work (MHC_ERR_UNSUPPORTED), so this runs without a GPU."""
    lib = mb.load()
    h = ctypes.c_void_p()
    p = mb.default_params()
    p.ordre_projection = 4                      # no such remap order
    assert lib.mhc_case_create(ctypes.byref(p), ctypes.byref(h)) == -3
    p = mb.default_params()
    p.projection_limiteur_id = 8                # no such limiter (TypesMahyco.h limiteur)
    assert lib.mhc_case_create(ctypes.byref(p), ctypes.byref(h)) == -3
    p = mb.default_params()
    p.projection_simple_pente = 1               # simple-pente without pente-borne: the reference stops
    assert lib.mhc_case_create(ctypes.byref(p), ctypes.byref(h)) == -3
    p.projection_pente_borne, p.ordre_projection = 1, 3   # pente-borne with the third-order remap
    assert lib.mhc_case_create(ctypes.byref(p), ctypes.byref(h)) == -3
    p = mb.default_params()
    p.env[0].elasto_model = 1
    p.is_euler_scheme = 2                       # elasto with a per-axis Euler remap
    assert lib.mhc_case_create(ctypes.byref(p), ctypes.byref(h)) == -3
    p.is_euler_scheme, p.projection_pente_borne = 0, 1   # elasto with pente-borne fluxes
    assert lib.mhc_case_create(ctypes.byref(p), ctypes.byref(h)) == -3
    p.projection_pente_borne, p.projection_limiteur_id = 0, 4   # ... or a generalised limiter
    assert lib.mhc_case_create(ctypes.byref(p), ctypes.byref(h)) == -3
    p.projection_limiteur_id = 0
    p.with_projection, p.nb_env = 0, 2          # elasto with two environments
    assert lib.mhc_case_create(ctypes.byref(p), ctypes.byref(h)) == -3
    p.env[0].elasto_model = 2                   # ... NewHypoModel too
    assert lib.mhc_case_create(ctypes.byref(p), ctypes.byref(h)) == -3
    p.nb_env, p.env[0].elasto_model = 1, 3      # no such elasto model
    assert lib.mhc_case_create(ctypes.byref(p), ctypes.byref(h)) == -3
    p = mb.default_params()
    p.is_euler_scheme = 1                       # is-euler-scheme NON
    assert lib.mhc_case_create(ctypes.byref(p), ctypes.byref(h)) == -3
    p.dim, p.is_euler_scheme = 2, 4             # per-axis Euler along z on a 2D mesh
    assert lib.mhc_case_create(ctypes.byref(p), ctypes.byref(h)) == -3
    p = mb.default_params()
    p.with_projection = 0
    mb.add_bc(p, "XMIN", "Density", 1.0)
    mb.add_bc(p, "XMAX", "GeometricPressure", 1.0)  # interleaved with a pressure surface
    assert lib.mhc_case_create(ctypes.byref(p), ctypes.byref(h)) == -3
    p = mb.default_params()
    p.is_euler_scheme = 3
    mb.add_bc(p, "XMIN", "Energy", 1.0)         # with a per-axis Euler remap
    assert lib.mhc_case_create(ctypes.byref(p), ctypes.byref(h)) == -3


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES", "x") != "" and os.path.exists("/dev/nvidia0"),
                    reason="a GPU is present")
def test_no_gpu_fails_loudly():
    p = mb.default_params()
    p.nx = p.ny = p.nz = 4
    with pytest.raises(mb.MahycoError):
        mb.Hydro(p)


def test_c_defaults_match_the_python_defaults():
    """mhc_case_params_default (for C / C++ hosts) writes the same reference
    defaults as mahyco_b200.case.default_params; host only, no GPU."""
    lib = mb.load()
    c = mb.CaseParams()
    ctypes.memset(ctypes.byref(c), 0xAB, ctypes.sizeof(c))
    lib.mhc_case_params_default(ctypes.byref(c))
    py = mb.default_params()
    assert bytes(c) == bytes(py)


def test_params_size_matches_the_binding():
    """The ctypes mirror of mhc_case_params has the library's layout size
    (host only, no GPU)."""
    lib = mb.load()
    assert lib.mhc_case_params_size() == ctypes.sizeof(mb.CaseParams)
