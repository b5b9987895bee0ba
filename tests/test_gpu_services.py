"""The per-method service surface and the field upload of the C ABI.

* Field upload (mhc_set_field): a state pushed onto the device by a host
  gives, after N iterations, the same fields bit for bit as the oracle given
  the same state through its own setter.
* IEquationOfState per method on the GPU against the known answers of
  tests/eos_kat.py (perfect gas, stiffened gas, Mie-Gruneisen): applyEOS,
  applyOneCellEOS with dp/de, initEOS, the getters, Endommagement.
* IRemap: appliRemap as sweeps + remapVariables equals the fused remap bit
  for bit; its argument checks and option getters.
* A compiled C++ host (tests/host/host_driver.cc, built by tests/host/
  Makefile) that drives the library through the C ABI alone -- defaults,
  upload, EOS per environment, the eleven entry points with the split
  remap, read-back -- matches the oracle given the same state.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from mahyco_b200.case import CaseParams, EOS_MIE_GRUNEISEN, EOS_PERFECT_GAS, EOS_STIFFENED_GAS
from tests import eos_kat
from tests.test_gpu_parity import compare

HERE = os.path.dirname(os.path.abspath(__file__))


def _bisod3d():
    from mahyco_b200.cases import sod, SUPERBEE
    return sod(dim=3, n=(24, 5, 4), L=(1.0, 0.2, 0.16), bi=True, limiter=SUPERBEE, deltat_init=1e-3)


@pytest.mark.gpu
def test_uploaded_state_matches_oracle_bitwise():
    from mahyco_b200 import Hydro
    from tests.oracle import Oracle
    p = _bisod3d()
    ora = Oracle(p, cr_pow=True)
    assert ora.init() == 0
    gpu = Hydro(p)
    gpu.hydroStartInit()
    rng = np.random.default_rng(5)
    # the host's state: per-environment energies and pressures of every
    # cell that holds the environment (mixed ones included), node
    # velocities, a global pseudo-viscosity
    for env in range(p.nb_env):
        for f in ("InternalEnergy", "Pressure"):
            v = ora.field(f, env) * (1.0 + 0.2 * rng.random(p.ncell))
            gpu.set_field(f, v, env)
            ora.set_field(f, v, env)
    vel = 0.02 * rng.standard_normal(3 * p.nnode)
    gpu.set_field("Velocity", vel)
    ora.set_field("Velocity", vel)
    q = 1e-3 * rng.random(p.ncell)
    gpu.set_field("PseudoViscosity", q)
    ora.set_field("PseudoViscosity", q)
    assert max(compare(gpu, ora, p.nb_env).values()) == 0.0
    n = 25
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


@pytest.mark.gpu
def test_uploaded_prescribed_velocities_advect_like_the_oracle():
    """sans-lagrange: the velocities at n (VelocityN, m_velocity_n) are the
    ones the node pass prescribes; a host field uploaded over the RIDER
    translation is advected bit for bit like the oracle's."""
    from mahyco_b200 import Hydro
    from mahyco_b200.cases import rider
    from tests.oracle import Oracle
    p = rider(31, n=(30, 30, 1))
    ora = Oracle(p, cr_pow=True)
    assert ora.init() == 0
    gpu = Hydro(p)
    gpu.hydroStartInit()
    assert np.array_equal(gpu.field("VelocityN"), ora.field("VelocityN"))
    xyz = ora.field("NodeCoord").reshape(-1, 3)
    v = np.zeros_like(xyz)
    v[:, 0], v[:, 1] = -(xyz[:, 1] - 0.5) * 3.0, (xyz[:, 0] - 0.5) * 3.0  # a solid rotation
    gpu.set_field("VelocityN", v.ravel())
    ora.set_field("VelocityN", v.ravel())
    n = 40
    gpu.cycle(n)
    assert gpu.synchronize() == 0
    assert ora.iterate(n) == 0
    errs = compare(gpu, ora, p.nb_env)
    errs["VelocityN"] = float(np.max(np.abs(gpu.field("VelocityN") - ora.field("VelocityN"))))
    gpu.close()
    bad = {k: v for k, v in errs.items() if v != 0.0}
    assert not bad, bad


@pytest.mark.gpu
def test_set_field_rejects_read_only_and_mid_iteration():
    import mahyco_b200 as mb
    h = mb.Hydro(_bisod3d())
    h.hydroStartInit()
    with pytest.raises(mb.MahycoError):
        h.set_field("NodeCoord", np.zeros(3 * h.nnode))
    with pytest.raises(mb.MahycoError):
        h.set_field("FracVol", np.ones(h.ncell))  # an environment field needs env >= 0
    h.saveValuesAtN()
    with pytest.raises(mb.MahycoError):  # between iterations only
        h.set_field("Density", np.ones(h.ncell))
    h.close()


def _one_env_case(eos, **env_kw):
    from mahyco_b200.cases import sod
    p = sod(dim=2, n=(8, 4), L=(1.0, 0.5), bi=False)
    p.nb_env = 1
    o = p.env[0]
    from mahyco_b200.case import env_defaults
    env_defaults(o, eos)
    for k, v in env_kw.items():
        setattr(o, k, v)
    o.densite_initiale, o.pression_initiale = env_kw.get("rho0", 1.0) or 1.0, 1.0
    return p


def _states(kind, n):
    base = {EOS_PERFECT_GAS: eos_kat.PG_STATES, EOS_STIFFENED_GAS: eos_kat.SG_STATES,
            EOS_MIE_GRUNEISEN: eos_kat.MG_STATES}[kind]
    rho = np.array([base[i % len(base)][0] for i in range(n)])
    e = np.array([base[i % len(base)][1] for i in range(n)])
    return rho, e


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [EOS_PERFECT_GAS, EOS_STIFFENED_GAS, EOS_MIE_GRUNEISEN])
def test_eos_methods_known_answers(kind):
    import mahyco_b200 as mb
    kw = {EOS_PERFECT_GAS: dict(adiabatic_cst=1.4),
          EOS_STIFFENED_GAS: dict(adiabatic_cst=4.4, limit_tension=6e8),
          EOS_MIE_GRUNEISEN: dict(rho0=2710.0, c0=5328.0, s1=1.338, gamma0=2.0)}[kind]
    p = _one_env_case(kind, **kw)
    o = p.env[0]
    h = mb.Hydro(p)
    h.hydroStartInit()
    assert h.getAdiabaticCst(0) == o.adiabatic_cst
    assert h.getdensityDamageThresold(0) == o.density_damage_thresold
    h.ReinitEOS(0)
    rho, e = _states(kind, p.ncell)
    h.set_field("Density", rho, 0)
    h.set_field("InternalEnergy", e, 0)
    h.eos_apply(0)  # applyEOS
    P, Cs = h.field("Pressure", 0), h.field("SoundSpeed", 0)
    for i in range(p.ncell):
        if kind == EOS_PERFECT_GAS:
            assert (P[i], Cs[i]) == eos_kat.pg_float(o.adiabatic_cst, rho[i], e[i])[:2], i
        elif kind == EOS_STIFFENED_GAS:
            assert (P[i], Cs[i]) == eos_kat.sg_float(o.adiabatic_cst, o.limit_tension, rho[i], e[i])[:2], i
        else:
            pe, _ = eos_kat.mg_exact(o, rho[i], e[i])
            assert abs(P[i] - float(pe)) <= 1e-13 * max(abs(float(pe)), 1e9), i
            assert eos_kat.rel(Cs[i], eos_kat.mg_sound_exact(o, rho[i], e[i])) <= 5e-6, i
    # applyOneCellEOS on one cell after changing its energy: p, c in place, dp/de back
    cell = 5
    e2 = e.copy()
    e2[cell] *= 1.5
    h.set_field("InternalEnergy", e2, 0)
    dpde = h.applyOneCellEOS(0, cell)
    P2, C2 = h.field("Pressure", 0), h.field("SoundSpeed", 0)
    assert np.array_equal(np.delete(P2, cell), np.delete(P, cell))  # only that cell changed
    if kind == EOS_PERFECT_GAS:
        assert (P2[cell], C2[cell], dpde) == eos_kat.pg_float(o.adiabatic_cst, rho[cell], e2[cell])
    elif kind == EOS_STIFFENED_GAS:
        assert (P2[cell], C2[cell], dpde) == eos_kat.sg_float(o.adiabatic_cst, o.limit_tension, rho[cell], e2[cell])
    else:
        _, de = eos_kat.mg_exact(o, rho[cell], e2[cell])
        assert eos_kat.rel(dpde, de) <= 1e-15
    # initEOS: energies and sound speeds back from pressure and density
    pin = np.linspace(1.0, 2.0, p.ncell) * (1e9 if kind != EOS_PERFECT_GAS else 1.0)
    h.set_field("Pressure", pin, 0)
    h.initEOS(0)
    E3, C3 = h.field("InternalEnergy", 0), h.field("SoundSpeed", 0)
    for i in range(p.ncell):
        if kind == EOS_PERFECT_GAS:
            assert (E3[i], C3[i]) == eos_kat.pg_init_float(o.adiabatic_cst, pin[i], rho[i]), i
        elif kind == EOS_STIFFENED_GAS:
            assert (E3[i], C3[i]) == eos_kat.sg_init_float(o.adiabatic_cst, o.limit_tension, pin[i], rho[i]), i
        else:
            assert (E3[i], C3[i]) == (pin[i] / o.gamma0, o.c0), i
    # Endommagement: nothing reaches the default thresholds ...
    h.Endommagement(0)
    assert h.synchronize() == 0
    # ... until a cell's pressure falls below tension-damage-thresold
    pin[3] = 2.0 * o.tension_damage_thresold
    h.set_field("Pressure", pin, 0)
    h.Endommagement(0)
    assert h.synchronize() & mb.ST_DAMAGE
    h.close()


@pytest.mark.gpu
def test_remap_split_equals_fused_remap():
    import mahyco_b200 as mb
    from mahyco_b200.cases import sedov
    p = sedov(dim=2, n=(16, 16), deltat_init=1e-4)
    a, b = mb.Hydro(p), mb.Hydro(p)
    a.hydroStartInit()
    b.hydroStartInit()
    assert b.getOrdreProjection() == p.ordre_projection
    assert not b.hasProjectionPenteBorne() and not b.hasProjectionSimplePente()
    assert not b.hasConservationEnergieTotale() and b.isEuler() == "Full"
    nvars = 18 * p.nb_env
    b.resizeRemapVariables(nvars, p.nb_env)
    with pytest.raises(mb.MahycoError):
        b.resizeRemapVariables(nvars + 1, p.nb_env)
    a.cycle(12)
    for it in range(12):
        for f in (b.saveValuesAtN, b.updateVelocity, b.applyBoundaryCondition, b.updatePosition,
                  b.computeGeometricValues, b.updateDensity, b.computeArtificialViscosity,
                  b.updateElasticityAndPlasticity, b.updateEnergyAndPressure):
            f()
        b.synchronizeUremap()
        if it % 2:
            b.remapSweeps()
            with pytest.raises(mb.MahycoError):  # the end of the time step needs remapVariables first
                b.computeDeltaT()
            b.remapVariables(p.dim, 1, nvars, p.nb_env)
        else:
            b.appliRemap(p.dim, 1, 3 * p.nb_env + 5, p.nb_env)
        b.computeDeltaT()
    assert a.synchronize() == 0 and b.synchronize() == 0
    for f in ("Density", "Pressure", "InternalEnergy", "Velocity", "NodeMass"):
        assert np.array_equal(a.field(f), b.field(f)), f
    assert a.scalars() == b.scalars()
    a.close()
    b.close()


@pytest.mark.gpu
def test_cpp_host_driver_matches_oracle(tmp_path):
    from tests.oracle import Oracle
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "host")], check=True)
    n = 30
    r = subprocess.run([os.path.join(HERE, "host", "_build", "host_driver"), str(tmp_path), str(n)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    words = r.stdout.split()
    assert words[0] == "ok" and int(words[1]) == n
    raw = (tmp_path / "params.bin").read_bytes()
    assert len(raw) == ctypes.sizeof(CaseParams)
    p = CaseParams.from_buffer_copy(raw)
    ora = Oracle(p, cr_pow=True)
    assert ora.init() == 0
    for env in range(p.nb_env):
        ora.set_field("InternalEnergy", np.fromfile(tmp_path / f"uploaded_InternalEnergy_{env}.bin"), env)
        ora.eos_apply(env)
    ora.set_field("Velocity", np.fromfile(tmp_path / "uploaded_Velocity_-1.bin"))
    assert ora.iterate(n) == 0
    assert float(words[2]) == ora.scalar("time") and float(words[3]) == ora.scalar("deltat")
    checked = 0
    for f in ("Density", "Pressure", "InternalEnergy", "SoundSpeed", "CellMass", "FracVol", "Velocity"):
        for env in range(-1, p.nb_env):
            path = tmp_path / f"result_{f}_{env}.bin"
            if not path.exists():
                continue
            got = np.fromfile(path)
            assert np.array_equal(got, ora.field(f, env)), (f, env)
            checked += 1
    assert checked >= 18


def _run_initial_fields_pair(p, fields, n):
    from mahyco_b200 import Hydro
    from tests.oracle import Oracle
    ora = Oracle(p, cr_pow=True)
    gpu = Hydro(p)
    for name, values in fields.items():
        ora.set_initial_field(name, values)
        gpu.set_initial_field(name, values)
    assert ora.init() == 0
    gpu.hydroStartInit()
    init = compare(gpu, ora, p.nb_env)
    gpu.cycle(n)
    st = gpu.synchronize()
    assert ora.iterate(n) == 0
    errs = compare(gpu, ora, p.nb_env)
    errs["NodeCoord"] = float(np.max(np.abs(gpu.field("NodeCoord") - ora.field("NodeCoord"))))
    gpu.close()
    return st, init, errs


@pytest.mark.gpu
def test_mesh_file_grid_matches_oracle_bitwise():
    """The Taylor bar of CAS_2D_Lag_Taylor_elasto on its Gmsh grid
    (plaqueTaylor.msh: node coordinates with the mesher's rounding, cells
    numbered column by column), EXTERNAL init with a user velocity,
    Mie-Gruneisen, elasto-plastic, anti-hourglass: the library equals the
    oracle bit for bit, plasticity included."""
    import json
    import os
    from mahyco_b200.case import params_from_dict
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "CAS_2D_Lag_Taylor_elasto.json")))
    p = params_from_dict(g["params"])
    assert p.mesh_cell_order == 1
    st, init, errs = _run_initial_fields_pair(p, g["init_fields"], 400)
    assert st == 0, st
    assert max(init.values()) == 0.0, init
    bad = {k: v for k, v in errs.items() if v != 0.0}
    assert not bad, bad


@pytest.mark.gpu
def test_external_initial_state_per_cell_matches_oracle_bitwise():
    """EXTERNAL case model with a per-cell <initialisation>: two groups of
    cells in two environments with their own density and pressure (a
    seeded patchwork), velocity 0; GPU and oracle bit for bit."""
    from mahyco_b200.cases import _external
    p = _external(velocity=(0.0, 0.0, 0.0))
    p.env[0].initialisation_utilisateur = 0
    p.nb_env = 2
    from mahyco_b200.case import env_defaults, EOS_STIFFENED_GAS
    env_defaults(p.env[1], EOS_STIFFENED_GAS)
    p.env[1].adiabatic_cst, p.env[1].limit_tension = 1.6, 0.05
    rng = np.random.default_rng(11)
    mat = (rng.random(p.ncell) < 0.4).astype(np.float64)
    rho = np.where(mat == 1.0, 2.0, 1.0) * (1.0 + 0.3 * rng.random(p.ncell))
    pre = np.where(mat == 1.0, 0.5, 1.0) * (1.0 + 0.3 * rng.random(p.ncell))
    st, init, errs = _run_initial_fields_pair(p, {"Materiau": mat, "Density": rho, "Pressure": pre}, 60)
    assert st == 0, st
    assert max(init.values()) == 0.0, init
    bad = {k: v for k, v in errs.items() if v != 0.0}
    assert not bad, bad
