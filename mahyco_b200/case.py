"""Case description: ctypes mirror of ``include/mahyco_case.h`` and a reader
for the subset of MaHyCo ``.arc`` datasets used by the hydro cycle.

Option names and defaults follow the reference descriptors:
``src/Mahyco.axl:263-557`` (module), ``src/Remap/RemapADI.axl:162-210``
(remap), ``src/eos/*/*.axl`` (equations of state) and
``src/time_history/EnvSummation.axl:27`` (time-history period).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import xml.etree.ElementTree as ET

MAX_ENV = 4
MAX_BC = 12
MAX_PTABLE = 32

EOS_PERFECT_GAS, EOS_STIFFENED_GAS, EOS_MIE_GRUNEISEN, EOS_FICTIF = 0, 1, 2, 3
EOS_BY_NAME = {"PerfectGas": EOS_PERFECT_GAS, "StiffenedGas": EOS_STIFFENED_GAS,
               "MieGruneisen": EOS_MIE_GRUNEISEN, "Fictif": EOS_FICTIF}
BC_BY_NAME = {"Vx": 0, "Vy": 1, "Vz": 2, "GeometricPressure": 3, "LinearPressure": 4, "Density": 5,
              "Energy": 6, "SuperGaussianEnergy": 7, "Pressure": 8, "SuperGaussianPressure": 9,
              "ContactHerzPressure": 10, "OFV": 11, "OnFilePressure": 12}
SURFACES = {"XMIN": 0, "YMIN": 1, "ZMIN": 2, "XMAX": 3, "YMAX": 4, "ZMAX": 5}
CASE_SOD, CASE_SEDOV, CASE_TWO_STATE, CASE_ONECELL, CASE_BUBBLES, CASE_RIDER, CASE_EXTERNAL = 1, 2, 3, 4, 5, 6, 7
CASE_TRIPLE_POINT = 8
CASE_BY_NAME = {"SOD": CASE_SOD, "SEDOV": CASE_SEDOV, "ONECELL": CASE_ONECELL, "CHOCBULLE": CASE_BUBBLES,
                "RIDER": CASE_RIDER, "EXTERNAL": CASE_EXTERNAL, "POINTTRIPLE": CASE_TRIPLE_POINT}
# RIDER cas-test ids (TypesMahyco.h:69-84): MonoRider* 23-30, Rider* 31-38
RIDER_TESTS = {n: 23 + i for i, n in enumerate(
    ("MonoRiderTx", "MonoRiderTy", "MonoRiderT45", "MonoRiderRotation", "MonoRiderVortex", "MonoRiderDeformation",
     "MonoRiderVortexTimeReverse", "MonoRiderDeformationTimeReverse", "RiderTx", "RiderTy", "RiderT45",
     "RiderRotation", "RiderVortex", "RiderDeformation", "RiderVortexTimeReverse",
     "RiderDeformationTimeReverse"))}
LENGTHS = {"racine-cubique-volume": 0, "faces-opposees": 1, "monodimX": 2,
           "monodimY": 3, "monodimZ": 4}
MINMOD, SUPERBEE, VANLEER = 0, 1, 2
MINMOD_G, SUPERBEE_G, VANLEER_G, ARITHMETIC_G, ULTRABEE_G = 3, 4, 5, 6, 7
DEPOT_NONE, DEPOT_CONSTANT, DEPOT_LINEAIRE, DEPOT_SUPER_GAUSSIAN = 0, 1, 2, 3
DEPOT_BY_NAME = {"DepotConstant": DEPOT_CONSTANT, "DepotLineaire": DEPOT_LINEAIRE,
                 "DepotSuperGaussian": DEPOT_SUPER_GAUSSIAN}
EULER_FULL, EULER_NONE, EULER_X, EULER_Y, EULER_Z = 0, 1, 2, 3, 4
EULER_BY_NAME = {"Full": EULER_FULL, "NON": EULER_NONE, "X": EULER_X, "Y": EULER_Y, "Z": EULER_Z}


class EnvParams(C.Structure):
    _fields_ = [
        ("eos", C.c_int),
        ("adiabatic_cst", C.c_double), ("limit_tension", C.c_double),
        ("specific_heat", C.c_double), ("tension_damage_thresold", C.c_double),
        ("density_damage_thresold", C.c_double),
        ("rho0", C.c_double), ("s1", C.c_double), ("s2", C.c_double), ("s3", C.c_double),
        ("gamma0", C.c_double), ("a", C.c_double), ("c0", C.c_double),
        ("energie_ref", C.c_double), ("temperature_ref", C.c_double),
        ("linear_pseudo_coeff", C.c_double), ("quadratic_pseudo_coeff", C.c_double),
        ("densite_initiale", C.c_double), ("pression_initiale", C.c_double),
        ("energie_initiale", C.c_double), ("temperature_initiale", C.c_double),
        ("vitesse_initiale", C.c_double * 3),
        ("elasto_model", C.c_int), ("rotation_order", C.c_int),
        ("shear_modulus", C.c_double), ("yield_strength", C.c_double),
        ("depot_type", C.c_int), ("depot_value", C.c_double), ("depot_origin", C.c_double * 3),
        ("depot_dependance", C.c_double * 4), ("depot_cutoff", C.c_double * 2),
        ("depot_tdebut", C.c_double), ("depot_tfin", C.c_double), ("depot_power", C.c_double),
        ("fictif_tdebut", C.c_double), ("fictif_tfin", C.c_double), ("fictif_p0", C.c_double),
        ("fictif_dpdt", C.c_double), ("initialisation_utilisateur", C.c_int),
    ]


class BC(C.Structure):
    _fields_ = [("kind", C.c_int), ("surface", C.c_int), ("value", C.c_double),
                ("tdebut", C.c_double), ("tfin", C.c_double), ("dependance", C.c_double * 4),
                ("cutoff", C.c_double * 2), ("power", C.c_double)]


class CaseParams(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("origin", C.c_double * 3), ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
        ("nb_env", C.c_int), ("env", EnvParams * MAX_ENV),
        ("cas_model", C.c_int), ("cas_test", C.c_int), ("sedov_energy", C.c_double),
        ("interface_pos", C.c_double), ("interface_dir", C.c_int),
        ("with_projection", C.c_int), ("pseudo_centree", C.c_int), ("with_newton", C.c_int),
        ("pression_explicite", C.c_int), ("deltat_constant", C.c_int),
        ("calcul_vitson_max", C.c_int), ("longueur_caracteristique", C.c_int),
        ("cfl", C.c_double), ("deltat_init", C.c_double), ("deltat_min", C.c_double),
        ("deltat_max", C.c_double), ("final_time", C.c_double), ("threshold", C.c_double),
        ("gravity", C.c_double * 3),
        ("nb_bc", C.c_int), ("bc", BC * MAX_BC),
        ("ordre_projection", C.c_int), ("projection_limiteur_id", C.c_int),
        ("is_euler_scheme", C.c_int), ("remap_threshold", C.c_double),
        ("time_history_period", C.c_int),
        ("coef_antiderive", C.c_double),
        ("projection_simple_pente", C.c_int),
        ("projection_pente_borne", C.c_int), ("projection_pente_borne_debar_fix", C.c_int),
        ("projection_pente_borne_mixte", C.c_int), ("projection_limiteur_pure_id", C.c_int),
        ("conservation_energie_totale", C.c_int),
        ("bubbles_n", C.c_int * 3), ("bubbles_first", C.c_double * 3), ("bubbles_delta", C.c_double * 3),
        ("bubbles_radius", C.c_double),
        ("sans_lagrange", C.c_int), ("rider_reverse", C.c_int), ("rider_parameter", C.c_double),
        ("rider_radius", C.c_double), ("rider_linear_density", C.c_int),
        ("schema_csts", C.c_int), ("mesh_cell_order", C.c_int),
        ("pressure_table_n", C.c_int), ("pressure_table_t", C.c_double * MAX_PTABLE),
        ("pressure_table_p", C.c_double * MAX_PTABLE),
    ]

    # -- convenience -------------------------------------------------------
    @property
    def ncell(self) -> int:
        return self.nx * self.ny * (self.nz if self.dim == 3 else 1)

    @property
    def nnode(self) -> int:
        return (self.nx + 1) * (self.ny + 1) * ((self.nz + 1) if self.dim == 3 else 1)


def env_defaults(e: EnvParams, eos: int = EOS_PERFECT_GAS) -> None:
    """Reference defaults of one ``<environment>`` block and its EOS service."""
    e.eos = eos
    e.adiabatic_cst = 1.4
    e.limit_tension = 0.01 if eos == EOS_STIFFENED_GAS else 0.0
    e.specific_heat = 921.0 if eos == EOS_MIE_GRUNEISEN else 0.0
    e.tension_damage_thresold = -1.0e12
    e.density_damage_thresold = 0.0
    e.rho0, e.s1, e.s2, e.s3 = 0.0, 1.4, 0.0, 0.0
    e.gamma0, e.a, e.c0 = 1.97, 0.48, 5240.0
    e.energie_ref, e.temperature_ref = 0.0, 300.0
    e.linear_pseudo_coeff, e.quadratic_pseudo_coeff = 0.5, 1.2
    e.densite_initiale, e.pression_initiale = 0.0, 1.0e5
    e.energie_initiale, e.temperature_initiale = 0.0, 0.0
    e.vitesse_initiale[:] = (0.0, 0.0, 0.0)
    e.elasto_model, e.rotation_order = 0, 1
    e.shear_modulus, e.yield_strength = 2.94e10, 3.0e8
    e.depot_type, e.depot_value = DEPOT_NONE, 0.0
    e.depot_origin[:] = (0.0, 0.0, 0.0)
    e.depot_dependance[:] = (0.0, 0.0, 0.0, 0.0)
    e.depot_cutoff[:] = (1000.0, 1000.0)
    e.depot_tdebut, e.depot_tfin = 0.0, 1000.0
    e.depot_power = 4.0


def default_params() -> CaseParams:
    """A CaseParams filled with the reference option defaults."""
    p = CaseParams()
    p.dim, p.nx, p.ny, p.nz = 3, 1, 1, 1
    p.origin[:] = (0.0, 0.0, 0.0)
    p.lx = p.ly = p.lz = 1.0
    p.nb_env = 1
    for i in range(MAX_ENV):
        env_defaults(p.env[i])
    p.cas_model, p.cas_test = CASE_SOD, 3
    p.sedov_energy = 0.244816
    p.interface_pos, p.interface_dir = 0.5, 0
    p.with_projection = 1
    p.pseudo_centree = 0
    p.with_newton = 0
    p.pression_explicite = 0
    p.deltat_constant = 0
    p.calcul_vitson_max = 1
    p.longueur_caracteristique = 0
    p.cfl, p.deltat_init, p.deltat_min, p.deltat_max = 0.3, 1.0e-5, 1.0e-8, 1.0e-2
    p.final_time = 1.0e30
    p.threshold = 1.0e-10
    p.gravity[:] = (0.0, 0.0, 0.0)
    p.nb_bc = 0
    for b in p.bc:
        b.cutoff[:] = (1000.0, 1000.0)
        b.power = 4.0
    p.ordre_projection = 2
    p.projection_limiteur_id = MINMOD
    p.is_euler_scheme = 0
    p.remap_threshold = 1.0e-10
    p.time_history_period = 10
    p.coef_antiderive = 0.0
    p.rider_radius = 0.15
    return p


def read_pressure_table(path: str) -> list[tuple[float, float]]:
    """(time, pressure) pairs of an OnFilePressure table: whitespace
    separated reals read two by two until the first that does not parse, as
    lireFichierCDL's stream loop does (MahycoAnnexe.cc:242-269)."""
    pairs, vals = [], []
    for tok in open(path).read().split():
        try:
            vals.append(float(tok))
        except ValueError:
            break
    for i in range(0, len(vals) - 1, 2):
        pairs.append((vals[i], vals[i + 1]))
    return pairs


def set_pressure_table(p: CaseParams, pairs) -> None:
    if len(pairs) > MAX_PTABLE:
        raise ValueError(f"at most {MAX_PTABLE} (time, pressure) pairs")
    p.pressure_table_n = len(pairs)
    for i, (t, v) in enumerate(pairs):
        p.pressure_table_t[i], p.pressure_table_p[i] = t, v


def add_bc(p: CaseParams, surface: str, kind: str, value: float = 0.0,
           tdebut: float = 0.0, tfin: float = 1000.0, dependance=(0.0, 0.0, 0.0, 0.0),
           cutoff=(1000.0, 1000.0), power: float = 4.0) -> None:
    if p.nb_bc >= MAX_BC:
        raise ValueError("too many boundary conditions")
    b = p.bc[p.nb_bc]
    b.kind, b.surface, b.value, b.tdebut, b.tfin = BC_BY_NAME[kind], SURFACES[surface], value, tdebut, tfin
    b.dependance[:] = dependance
    b.cutoff[:] = cutoff
    b.power = power
    p.nb_bc += 1


def symmetry_bcs(p: CaseParams, surfaces=("XMIN", "XMAX", "YMIN", "YMAX", "ZMIN", "ZMAX")) -> None:
    """Zero normal velocity on the given faces, as the reference datasets set it."""
    for s in surfaces:
        add_bc(p, s, {"X": "Vx", "Y": "Vy", "Z": "Vz"}[s[0]], 0.0)


# ---------------------------------------------------------------------------
# .arc reader
# ---------------------------------------------------------------------------
def _txt(node, tag, default=None, conv=float):
    el = node.find(tag)
    if el is None or el.text is None or not el.text.strip():
        return default
    return conv(el.text.strip())


def _bool(s: str) -> bool:
    return s.strip().lower() in ("1", "true", "yes")


def read_arc(path: str) -> tuple[CaseParams, dict]:
    """Parse a MaHyCo ``Donnees.arc`` into CaseParams.

    Returns ``(params, info)`` where ``info`` holds environment names, the
    time loop, the post-processed and EnvSummation variable lists and
    anything the hot path ignores.  Unsupported options that change the cycle
    (elasto models other than DefaultModel,
    super-Gaussian energy deposits, non-velocity boundary conditions) raise
    ``NotImplementedError``.
    """
    root = ET.parse(path).getroot()
    p = default_params()
    info: dict = {"env_names": [], "timeloop": None}
    tl = root.find("arcane/timeloop")
    info["timeloop"] = tl.text.strip() if tl is not None else "MahycoLoop"
    # post-processed variables (Ensight) and EnvSummation variables
    info["output_vars"] = [v.text.strip() for v in root.findall("arcane-post-processing/output/variable")]
    info["history_vars"] = [v.text.strip() for v in root.findall("time-history/bilan/variable")]
    # save-init: the post-processing also writes the initial state (step 0)
    info["save_init"] = bool(_txt(root, "arcane-post-processing/save-init", False, _bool))
    cart = root.find("mesh/meshgenerator/cartesian")
    mfile = root.find("mesh/file")
    info["init_fields"] = {}
    msh = None
    if cart is None and mfile is not None and mfile.text.strip().endswith(".msh"):
        # a Gmsh file of logically structured quadrangles, 2D: its node
        # coordinates and the <initialisation> values of its cell groups
        # are the case's initial fields (mahyco_b200.msh)
        from .msh import read_msh
        msh = read_msh(os.path.join(os.path.dirname(os.path.abspath(path)), mfile.text.strip()))
        xyz = msh["coords"]
        p.dim, p.nx, p.ny, p.nz = 2, msh["nx"], msh["ny"], 1
        p.origin[:] = (float(xyz[:, 0].min()), float(xyz[:, 1].min()), 0.0)
        p.lx, p.ly, p.lz = float(xyz[:, 0].max() - xyz[:, 0].min()), float(xyz[:, 1].max() - xyz[:, 1].min()), 0.0
        info["init_fields"]["NodeCoord"] = xyz.ravel().tolist()
        info["msh_sides"] = msh["sides"]
        info["mesh_file"] = msh["file_order"]
        # the file's elements run column by column: its sums over cells too
        order = msh["cell_order"]
        nx_, ny_ = msh["nx"], msh["ny"]
        colmajor = all(order[a + nx_ * b] == a * ny_ + b for a in range(nx_) for b in range(ny_))
        rowmajor = all(order[c] == c for c in range(nx_ * ny_))
        if not (colmajor or rowmajor):
            raise NotImplementedError("mesh file cells neither row by row nor column by column")
        p.mesh_cell_order = 1 if colmajor and not rowmajor else 0
        vals: dict[str, dict[str, float]] = {}
        for v in root.findall("mesh/initialisation/variable"):
            vals.setdefault(v.get("nom"), {})[v.get("groupe")] = float(v.get("valeur"))
        for var in ("Materiau", "Density", "Pressure"):
            if var in vals:
                per_group = vals[var]
                missing = {g for g in msh["cell_groups"] if g not in per_group}
                if missing:
                    raise NotImplementedError(f"{var} not initialised on cell groups {sorted(missing)}")
                info["init_fields"][var] = [per_group[g] for g in msh["cell_groups"]]
    elif cart is None:
        raise NotImplementedError("only the cartesian mesh generator and Gmsh quadrangle files are supported")
    if msh is not None:
        org = None
    else:
        org = [float(v) for v in cart.find("origine").text.split()]
    if msh is None:
        p.origin[:] = (org + [0.0, 0.0, 0.0])[:3]
        lx, ly, lz = cart.find("lx"), cart.find("ly"), cart.find("lz")
        p.lx, p.nx = float(lx.text), int(lx.get("nx"))
        p.ly, p.ny = float(ly.text), int(ly.get("ny"))
        if lz is not None:
            p.dim, p.lz, p.nz = 3, float(lz.text), int(lz.get("nz"))
        else:
            p.dim, p.lz, p.nz = 2, 0.0, 1
        for el, n in ((lx, "prx"), (ly, "pry"), (lz, "prz")):
            if el is not None and float(el.get(n, "1.0")) != 1.0:
                raise NotImplementedError("non-uniform cartesian progression")
    m = root.find("mahyco")
    envs = m.findall("environment")
    if not 1 <= len(envs) <= MAX_ENV:
        raise NotImplementedError("1..4 environments supported")
    p.nb_env = len(envs)
    for i, ev in enumerate(envs):
        info["env_names"].append(ev.find("name").text.strip())
        eosel = ev.find("eos-model")
        kind = EOS_BY_NAME[eosel.get("name")]
        e = p.env[i]
        env_defaults(e, kind)
        e.densite_initiale = _txt(ev, "densite-initiale", 0.0)
        e.pression_initiale = _txt(ev, "pression-initiale", 1.0e5)
        e.energie_initiale = _txt(ev, "energie-initiale", 0.0)
        e.temperature_initiale = _txt(ev, "temperature-initiale", 0.0)
        vi = ev.find("vitesse-initiale")
        if vi is not None:
            e.vitesse_initiale[:] = [float(v) for v in vi.text.split()]
        e.initialisation_utilisateur = int(_txt(ev, "initialisation-utilisateur", False, _bool))
        e.linear_pseudo_coeff = _txt(ev, "linear-pseudo-coeff", 0.5)
        e.quadratic_pseudo_coeff = _txt(ev, "quadratic-pseudo-coeff", 1.2)
        for tag, attr in (("adiabatic-cst", "adiabatic_cst"), ("limit-tension", "limit_tension"),
                          ("specific-heat", "specific_heat"), ("rho0", "rho0"), ("s1", "s1"),
                          ("s2", "s2"), ("s3", "s3"), ("gamma0", "gamma0"), ("a", "a"), ("c0", "c0"),
                          ("energie-ref", "energie_ref"), ("temperature-ref", "temperature_ref"),
                          ("tension-damage-thresold", "tension_damage_thresold"),
                          ("density-damage-thresold", "density_damage_thresold"),
                          ("tdebut-pression", "fictif_tdebut"), ("tfin-pression", "fictif_tfin"),
                          ("valeur-debut-pression", "fictif_p0"),
                          ("valeur-dependance-temps", "fictif_dpdt")):
            v = _txt(eosel, tag, None)
            if v is not None:
                setattr(e, attr, v)
        el = ev.find("elasto-model")
        if el is not None and el.get("name") not in (None, "NoModel"):
            if el.get("name") not in ("DefaultModel", "NewHypoModel"):
                raise NotImplementedError(f"elasto-model {el.get('name')}")
            mu_el, y_el = el.find("elasto-mu-model"), el.find("elasto-y-model")
            if (mu_el is not None and mu_el.get("name", "EPP") != "EPP") or \
                    (y_el is not None and y_el.get("name", "YEPP") != "YEPP"):
                raise NotImplementedError("elasto mu/y models other than EPP/YEPP")
            e.elasto_model = 2 if el.get("name") == "NewHypoModel" else 1
            e.rotation_order = _txt(el, "ordre-rotation", 1, int)
            if mu_el is not None:
                e.shear_modulus = _txt(mu_el, "elastic-cst", 2.94e10)
            if y_el is not None:
                e.yield_strength = _txt(y_el, "limit-elastic", 3.0e8)
        dep = ev.find("energy-depot")
        if dep is not None:
            kind = _txt(dep, "type", "DepotConstant", str)
            if kind not in DEPOT_BY_NAME:
                raise NotImplementedError(f"energy deposit {kind}")
            e.depot_type = DEPOT_BY_NAME[kind]
            e.depot_power = _txt(dep, "power", 4.0)
            e.depot_value = _txt(dep, "valeur-source-energie", 0.0)
            org = _txt(dep, "origine", "0. 0. 0.", str).split()
            e.depot_origin[:] = [float(v) for v in org]
            e.depot_dependance[:] = [_txt(dep, t, 0.0) for t in ("dependanceX", "dependanceY", "dependanceZ",
                                                                  "dependanceT")]
            e.depot_cutoff[:] = (_txt(dep, "cutoffX", 1000.0), _txt(dep, "cutoffY", 1000.0))
            e.depot_tdebut, e.depot_tfin = _txt(dep, "Tdebut", 0.0), _txt(dep, "Tfin", 1000.0)
    cm = m.find("cas-model")
    if cm is None:
        # the default cas-model (Mahyco.axl:386): EXTERNAL
        cm = ET.Element("cas-model", {"name": "EXTERNAL"})
    p.cas_model = CASE_BY_NAME[cm.get("name")]
    p.cas_test = _txt(cm, "cas-test", 0, int)
    if p.cas_model == CASE_BUBBLES:
        # the lattice of CHOCBULLE (src/casTest/CHOCBULLE/CHOCBULLE.axl:180-202);
        # its random and file-read bubbles and fictitious regions are not read
        if _txt(cm, "nombre-bulles-aleatoires", 0, int) or cm.find("fichier-bulles") is not None:
            raise NotImplementedError("CHOCBULLE: random or file-read bubbles")
        p.bubbles_n[:] = [_txt(cm, f"nombre-bulles-{a}", 1 if a == "z" else 0, int) for a in "xyz"]
        p.bubbles_first[:] = [float(v) for v in _txt(cm, "position-premiere-bulle", "0. 0. 0.", str).split()]
        p.bubbles_delta[:] = [_txt(cm, f"delta{a}-bulle", 0.0) for a in "xyz"]
        p.bubbles_radius = _txt(cm, "rayon-bulle", 0.0)
    if p.cas_model == CASE_RIDER:
        # RIDER.axl:145-166
        p.rider_reverse = int(_txt(cm, "reverse-option", False, _bool))
        p.rider_parameter = _txt(cm, "parametre", 0.0)
        p.rider_radius = _txt(cm, "rayon-bulle", 0.15)
        p.rider_linear_density = int(_txt(cm, "densite-interieure-initiale-lineaire", False, _bool))
    rm = m.find("remap")
    if rm is not None:
        if rm.get("name", "RemapADI") != "RemapADI":
            raise NotImplementedError("only the RemapADI service")
        p.ordre_projection = _txt(rm, "ordre-projection", 2, int)
        p.projection_limiteur_id = _txt(rm, "projection-limiteur-id", 0, int)
        p.remap_threshold = _txt(rm, "threshold", 1.0e-10)
        eul = _txt(rm, "is-euler-scheme", "Full", str)
        if eul not in EULER_BY_NAME or eul == "NON":
            raise NotImplementedError(f"is-euler-scheme {eul}")
        p.is_euler_scheme = EULER_BY_NAME[eul]
        p.conservation_energie_totale = int(_txt(rm, "conservation-energie-totale", False, _bool))
        p.projection_simple_pente = int(_txt(rm, "projection-simple-pente", False, _bool))
        p.projection_pente_borne = int(_txt(rm, "projection-pente-borne", False, _bool))
        p.projection_pente_borne_debar_fix = _txt(rm, "projection-pente-borne-debar-fix", 0, int)
        p.projection_pente_borne_mixte = int(_txt(rm, "projection-pente-borne-mixte", False, _bool))
        p.projection_limiteur_pure_id = _txt(rm, "projection-limiteur-pure-id", 0, int)
        if p.ordre_projection not in (1, 2, 3) or not 0 <= p.projection_limiteur_id <= 7:
            raise NotImplementedError("ordre-projection / projection-limiteur-id out of range")
    p.schema_csts = int(_txt(m, "schema-csts", False, _bool))
    p.sans_lagrange = int(_txt(m, "sans-lagrange", False, _bool))
    p.pseudo_centree = int(_txt(m, "pseudo-centree", False, _bool))
    p.with_projection = int(_txt(m, "with-projection", True, _bool))
    if info["timeloop"] == "MahycoLagrangeLoop":
        p.with_projection = 0
    p.with_newton = int(_txt(m, "with-newton", False, _bool))
    p.pression_explicite = int(_txt(m, "pression-explicite", False, _bool))
    p.deltat_constant = int(_txt(m, "deltat-constant", False, _bool))
    p.calcul_vitson_max = int(_txt(m, "calcul-vitson-max", True, _bool))
    p.longueur_caracteristique = LENGTHS[_txt(m, "longueur-caracteristique", "racine-cubique-volume", str)]
    p.cfl = _txt(m, "cfl", 0.3)
    p.deltat_init = _txt(m, "deltat-init", 1.0e-5)
    p.deltat_min = _txt(m, "deltat-min", 1.0e-8)
    p.deltat_max = _txt(m, "deltat-max", 1.0e-2)
    p.final_time = _txt(m, "final-time", 1.0)
    p.threshold = _txt(m, "threshold", 1.0e-10)
    g = m.find("gravity")
    if g is not None:
        p.gravity[:] = [float(v) for v in g.text.split()]
    p.coef_antiderive = _txt(m, "coef-antiderive", 0.0)
    for b in m.findall("boundary-condition"):
        kind = b.find("type").text.strip()
        if kind not in BC_BY_NAME:
            raise NotImplementedError(f"boundary condition {kind}")
        surf = b.find("surface").text.strip()
        if msh is not None:
            # a mesh file's boundary group: the logical side it lies on
            if surf not in msh["sides"]:
                raise NotImplementedError(f"boundary group {surf} is not one side of the grid")
            surf = {v: k for k, v in SURFACES.items()}[msh["sides"][surf]]
        add_bc(p, surf, kind, _txt(b, "value", 0.0),
               _txt(b, "Tdebut", 0.0), _txt(b, "Tfin", 1000.0),
               tuple(_txt(b, t, 0.0) for t in ("dependanceX", "dependanceY", "dependanceZ", "dependanceT")),
               (_txt(b, "cutoffX", 1000.0), _txt(b, "cutoffY", 1000.0)), _txt(b, "power", 4.0))
        if kind == "OnFilePressure" and p.pressure_table_n == 0:
            # the reference reads Pression.data from the run directory
            # whatever the fichier option says (MahycoModule.cc:77-82)
            fn = os.path.join(os.path.dirname(os.path.abspath(path)), "Pression.data")
            if os.path.exists(fn):
                set_pressure_table(p, read_pressure_table(fn))
    th = root.find("time-history/bilan")
    if th is not None:
        p.time_history_period = _txt(th, "periode", 10, int)
    # Arcane records history values only every output-history-period
    # iterations: EnvSummation lines come out at multiples of both periods
    ohp = _txt(root.find("arcane-post-processing"), "output-history-period", 1, int) \
        if root.find("arcane-post-processing") is not None else 1
    if ohp > 1:
        p.time_history_period = math.lcm(p.time_history_period if p.time_history_period > 0 else 10, ohp)
    return p, info


# ---------------------------------------------------------------------------
# (de)serialisation
# ---------------------------------------------------------------------------
def _to_py(v):
    if isinstance(v, C.Array):
        return [_to_py(x) for x in v]
    if isinstance(v, C.Structure):
        return {n: _to_py(getattr(v, n)) for n, _ in v._fields_}
    return v


def _from_py(obj, v):
    for n, _ in obj._fields_:
        if n not in v:
            continue
        cur = getattr(obj, n)
        if isinstance(cur, C.Array):
            for i, x in enumerate(v[n]):
                if isinstance(cur[i], C.Structure):
                    _from_py(cur[i], x)
                else:
                    cur[i] = x
        elif isinstance(cur, C.Structure):
            _from_py(cur, v[n])
        else:
            setattr(obj, n, v[n])


def params_to_dict(p: CaseParams) -> dict:
    return _to_py(p)


def params_from_dict(d: dict) -> CaseParams:
    p = default_params()
    _from_py(p, d)
    return p
