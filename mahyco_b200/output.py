"""Outputs in the reference's formats, and a driver that runs a dataset.

A NONREGRESSION dataset run through this library writes the same files as
the reference, so the reference's own comparison (``diff -r`` of
``output/depouillement`` and ``output/courbes/gnuplot``,
NONREGRESSION/launch_test.sh:74-96) applies unchanged:

* EnvSummation time histories (src/time_history/EnvSummationService.cc:77-169):
  ``output/courbes/gnuplot/<Variable>_<Environment>``, one ``time value``
  line per period-th iteration, 17 significant digits;
* Ensight gold ASCII of the final state (Arcane's post-processing service):
  ``output/depouillement/ensight.case``, ``ensight.geo/ensight.geo000000``
  and ``<Variable>/<Variable>000000``, values with 6 significant digits;
  with ``save-init`` the initial state is step 000000 and the final one
  step 000001.
"""
from __future__ import annotations

import os

import numpy as np

from .case import CaseParams, read_arc

HISTORY_VARS = ("CellMass", "Pressure", "Density", "InternalEnergy")
NODE_VARS = {"Velocity": "vector", "NodeMass": "scalar", "NodeCoord": "vector"}
# post-processed variables the Ensight writer produces; the others of a
# dataset's <output> list are left out
ENSIGHT_VARS = frozenset({"CellMass", "Pressure", "Density", "Velocity", "NodeMass", "InternalEnergy",
                          "PseudoViscosity", "Materiau", "SoundSpeed", "CellVolume", "StrainTensorXX",
                          "StrainTensorYY", "StrainTensorXY", "StrainTensorXZ", "StrainTensorYZ",
                          "Temperature", "PlasticDeformation", "PlasticDeformationVelocity", "StrainNorm",
                          "FracPhase1", "FracPhase2", "FracPhase3"})


def frac_phase(h, var: str) -> np.ndarray:
    """The phase fractions of the cells: only the tabulated EOS (not built)
    changes them; ONECELL sets the first to 1 (ONECELLService.cc:29-31),
    the other initialisations leave the 0 of hydroStartInit."""
    from .case import CASE_ONECELL
    one = var == "FracPhase1" and h.params.cas_model == CASE_ONECELL
    return np.full(h.ncell, 1.0 if one else 0.0)


def write_gnuplot(out_dir: str, env_names: list[str], rows: np.ndarray, variables=HISTORY_VARS) -> list[str]:
    """EnvSummation curves: ``rows`` holds one mhc_time_history line per
    recorded iteration (time, then per environment CellMass, Pressure,
    Density, InternalEnergy, presence).  Returns the files written."""
    d = os.path.join(out_dir, "courbes", "gnuplot")
    os.makedirs(d, exist_ok=True)
    written = []
    for e, env in enumerate(env_names):
        for q, var in enumerate(HISTORY_VARS):
            if var not in variables:
                continue
            lines = [f"{r[0]:.16E} {r[1 + 5 * e + q]:.16E}\n" for r in rows if r[1 + 5 * e + 4] != 0.]
            if not lines:
                continue
            fn = os.path.join(d, f"{var}_{env}")
            with open(fn, "w") as f:
                f.writelines(lines)
            written.append(fn)
    return written


def _values(a: np.ndarray) -> str:
    return "".join(f"{v:12.5e}\n" for v in a)


def materiau(h) -> np.ndarray:
    """The Materiau cell variable: sum over environments of index x volume
    fraction (PrepareRemap.cc:227-235); a pure cell holds its environment's
    index."""
    p: CaseParams = h.params
    mask = h.field("EnvMask").astype(np.int64)
    out = np.zeros(h.ncell)
    pure = (mask & (mask - 1)) == 0
    for e in range(p.nb_env):
        has = (mask >> e) & 1
        if p.nb_env > 1:
            f = h.field("FracVol", e)
            out += np.where(pure, 0., e * f * has)
        out += np.where(pure & (has == 1), float(e), 0.)
    return out


def write_ensight(h, out_dir: str, variables: list[str], time: float, step: int = 0,
                  times: list[float] | None = None, mesh_file: dict | None = None) -> list[str]:
    """Ensight gold ASCII files of the current state of case ``h`` as time
    step ``step``; ``times`` (default ``[time]``) are the time values of
    every step written so far, listed in ensight.case.  Variables outside
    ENSIGHT_VARS are skipped.  ``mesh_file`` (``read_msh``'s ``file_order``)
    writes a Gmsh grid's nodes, quadrangles and values in the file's
    numbering, as the reference does."""
    times = [time] if times is None else times
    variables = [v for v in variables if v in ENSIGHT_VARS]
    sfx = f"{step:06d}"
    p: CaseParams = h.params
    d = os.path.join(out_dir, "depouillement")
    os.makedirs(os.path.join(d, "ensight.geo"), exist_ok=True)
    dim = p.dim
    nx, ny, nz = p.nx, p.ny, (p.nz if dim == 3 else 1)
    nnx, nny, nnz = nx + 1, ny + 1, (nz + 1 if dim == 3 else 1)
    nn = h.nnode
    if p.with_projection and p.is_euler_scheme == 0:
        # Full Euler scheme: the mesh is back on the initial grid
        a, b, c = np.meshgrid(np.arange(nnx), np.arange(nny), np.arange(nnz), indexing="ij")
        a, b, c = (t.transpose(2, 1, 0).ravel() for t in (a, b, c))
        xs = p.origin[0] + a * (p.lx / p.nx)
        ys = p.origin[1] + b * (p.ly / p.ny)
        zs = p.origin[2] + c * (p.lz / p.nz) if dim == 3 else np.zeros(nn)
    else:
        # Lagrangian run, or per-axis Euler (the remapped axis is on the
        # initial grid, the others Lagrangian)
        xyz = h.field("NodeCoord").reshape(-1, 3)
        xs, ys, zs = xyz[:, 0], xyz[:, 1], xyz[:, 2] if dim == 3 else np.zeros(nn)
    written = []
    # geometry: node coordinates (x, y, z blocks) and 1-based connectivity
    etype = "hexa8" if dim == 3 else "quad4"
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = (a.transpose(2, 1, 0).ravel() for a in (i, j, k))
    nid = lambda a, b, c: 1 + a + nnx * (b + nny * c)
    offs = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0)]
    if dim == 3:
        offs += [(0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    conn = np.stack([nid(i + a, j + b, k + c) for a, b, c in offs], axis=1)
    cell_perm = node_perm = None
    if mesh_file is not None:
        cell_perm = np.asarray(mesh_file["cells"])
        node_perm = np.asarray(mesh_file["nodes"])
        xs, ys, zs = xs[node_perm], ys[node_perm], zs[node_perm]
        conn = np.asarray(mesh_file["conn"])
        nn = len(node_perm)
    geo = ["Output ensight test\n", "File description\n", "node id assign\n", "element id assign\n",
           "part\n", f"{1:10d}\n", "AllCells\n", "coordinates\n", f"{nn:10d}\n",
           _values(xs), _values(ys), _values(zs), f"{etype}\n", f"{h.ncell:10d}\n",
           "".join("".join(f"{v:10d}" for v in row) + "\n" for row in conn)]
    fn = os.path.join(d, "ensight.geo", "ensight.geo" + sfx)
    with open(fn, "w") as f:
        f.writelines(geo)
    written.append(fn)
    entries = []
    for var in variables:
        if var in NODE_VARS:
            kind = NODE_VARS[var]
            a = h.field(var)
            if kind == "scalar":
                body = _values(a if node_perm is None else a[node_perm])
            else:
                v = a.reshape(-1, 3)
                if node_perm is not None:
                    v = v[node_perm]
                body = _values(v[:, 0]) + _values(v[:, 1]) + _values(v[:, 2])
            text = f"{var}\npart\n{1:10d}\ncoordinates\n" + body
            entries.append(f"{kind} per node:       1   {var} {var}/{var}******\n")
        else:
            if var == "Materiau":
                a = materiau(h)
            elif var.startswith("FracPhase"):
                a = frac_phase(h, var)
            else:
                a = h.field(var)
            if cell_perm is not None:
                a = a[cell_perm]
            text = f"{var}\npart\n{1:10d}\n{etype}\n" + _values(a)
            entries.append(f"scalar per element:    1   {var} {var}/{var}******\n")
        os.makedirs(os.path.join(d, var), exist_ok=True)
        fn = os.path.join(d, var, f"{var}{sfx}")
        with open(fn, "w") as f:
            f.write(text)
        written.append(fn)
    case = ["FORMAT\n", "type: ensight gold\n", "\n", "GEOMETRY\n", "model: 1 ensight.geo/ensight.geo******\n",
            "\n", "VARIABLE\n", *entries, "\n", "TIME\n", "time set:              1\n",
            f"number of steps:       {len(times)}\n", "filename start number: 0\n", "filename increment:    1\n",
            "time values:\n", *(f"{t:.15g}\n" for t in times), "\n"]
    fn = os.path.join(d, "ensight.case")
    with open(fn, "w") as f:
        f.writelines(case)
    written.append(fn)
    return written


def run_arc(arc_path: str, out_dir: str, max_iter: int = 10 ** 7) -> dict:
    """Run a Donnees.arc to its final time on the GPU and write the
    reference's outputs (EnvSummation curves, final Ensight state) under
    ``out_dir``.  Returns the final scalars and the files written."""
    p, info = read_arc(arc_path)
    return run_case(p, info, out_dir, max_iter)


def run_case(p: CaseParams, info: dict, out_dir: str, max_iter: int = 10 ** 7) -> dict:
    """run_arc on parameters already read (``info``: env_names and,
    optionally, output_vars, history_vars and save_init as read_arc returns
    them)."""
    from . import Hydro, ST_STOP
    period = p.time_history_period if p.time_history_period > 0 else 10
    h = Hydro(p)
    try:
        for name, values in info.get("init_fields", {}).items():
            h.set_initial_field(name, values)
        h.hydroStartInit()
        init_files = []
        mf = info.get("mesh_file")
        if info.get("save_init"):
            init_files = write_ensight(h, out_dir, info.get("output_vars", []), 0.0, mesh_file=mf)
        rows = []
        it = 0
        st = 0
        while it < max_iter:
            h.cycle(1)
            st = h.synchronize()
            it += 1
            if st not in (0, ST_STOP):
                break
            if it % period == 0:
                rows.append(h.time_history())
            if st == ST_STOP:
                break
        s = h.scalars()
        files = write_gnuplot(out_dir, info["env_names"], np.array(rows), info.get("history_vars", HISTORY_VARS))
        if info.get("save_init"):
            files += init_files + write_ensight(h, out_dir, info.get("output_vars", []), s["time"], 1,
                                                [0.0, s["time"]], mesh_file=mf)
        else:
            files += write_ensight(h, out_dir, info.get("output_vars", []), s["time"], mesh_file=mf)
        return {"scalars": s, "files": files}
    finally:
        h.close()
