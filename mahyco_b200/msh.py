"""Gmsh 4.1 ASCII meshes of logically structured quadrangles.

The reference reads ``<mesh><file>X.msh</file>`` through Arcane's mesh
readers (``NONREGRESSION/CAS_2D_Lag_Taylor_elasto``,
``CAS_2D_Lag_SodCaseX_msh``, ``CAS_2D_Lag_NOH``).  Those meshes are
transfinite grids of quadrangles whose nodes carry the mesher's rounding
(a column of a uniform grid at x = 0.0004 reads 0.000399999999999,
0.0004 or 0.000400000000001).  This reader recovers their (i, j)
structure from the connectivity, so that the structured kernels run them
with the file's exact node coordinates:

* every quadrangle lists its nodes counter-clockwise from its (i, j)
  corner: (i, j), (i+1, j), (i+1, j+1), (i, j+1);
* the grid is numbered like the library's (cells x-fastest, nodes
  (nx + 1)-fastest);
* each 2D physical group names cells (an ``<initialisation>`` group of the
  dataset), each 1D physical group a side of the logical rectangle (a
  boundary-condition surface of the dataset).
"""
from __future__ import annotations

import collections

import numpy as np

# logical sides, numbered like mhc_surface (include/mahyco_case.h)
SIDES = {"i=0": 0, "j=0": 1, "i=nx": 3, "j=ny": 4}


def _sections(text: str) -> dict[str, list[str]]:
    out: dict[str, list[str]] = {}
    lines = text.split("\n")
    i = 0
    while i < len(lines):
        s = lines[i].strip()
        if s.startswith("$") and not s.startswith("$End"):
            name = s[1:]
            j = i + 1
            while lines[j].strip() != "$End" + name:
                j += 1
            out[name] = [l for l in lines[i + 1:j]]
            i = j
        i += 1
    return out


def read_msh(path: str) -> dict:
    """The structured view of a Gmsh 4.1 ASCII quadrangle mesh: ``nx``,
    ``ny``, ``coords`` ((nx+1)(ny+1) x 3, library node order),
    ``cell_groups`` (the 2D physical group name of every cell, library
    cell order), ``sides`` (1D physical group name -> logical side, an
    mhc_surface number), ``cell_order`` (the file's element index of every
    library cell), ``node_tags`` (the file's node tag of every library
    node) and ``file_order``, the numbering the reference's outputs use
    (its mesh reader numbers the quadrangles and the nodes they use in
    file order): ``cells`` (the library cell of every quadrangle),
    ``nodes`` (the library node of every used node) and ``conn`` (every
    quadrangle's nodes as 1-based positions in ``nodes``).  Raises
    NotImplementedError when the mesh is not a logically structured grid of
    quadrangles."""
    sec = _sections(open(path).read())
    fmt = sec["MeshFormat"][0].split()
    if not fmt[0].startswith("4") or fmt[1] != "0":
        raise NotImplementedError("only Gmsh 4.x ASCII meshes")
    names = {}
    if "PhysicalNames" in sec:
        for l in sec["PhysicalNames"][1:]:
            if not l.strip():
                continue
            d, tag, name = l.split(maxsplit=2)
            names[(int(d), int(tag))] = name.strip().strip('"')
    # entity -> physical tags
    ent_phys: dict[tuple[int, int], list[int]] = {}
    ent = [l for l in sec.get("Entities", []) if l.strip()]
    if ent:
        counts = list(map(int, ent[0].split()))
        row = 1
        for d in range(4):
            for _ in range(counts[d]):
                v = ent[row].split()
                row += 1
                tag = int(v[0])
                if d == 0:
                    np_ = int(v[4]); phys = [int(x) for x in v[5:5 + np_]]
                else:
                    np_ = int(v[7]); phys = [int(x) for x in v[8:8 + np_]]
                ent_phys[(d, tag)] = phys
    # nodes
    nl = [l for l in sec["Nodes"] if l.strip()]
    nblocks = int(nl[0].split()[0])
    coords: dict[int, tuple[float, float, float]] = {}
    file_nodes: list[int] = []
    r = 1
    for _ in range(nblocks):
        d, tag, param, n = map(int, nl[r].split())
        r += 1
        tags = [int(nl[r + k]) for k in range(n)]
        file_nodes += tags
        r += n
        for k in range(n):
            x, y, z = (float(t) for t in nl[r + k].split()[:3])
            coords[tags[k]] = (x, y, z)
        r += n
    # elements
    el = [l for l in sec["Elements"] if l.strip()]
    nblocks = int(el[0].split()[0])
    quads, lines = [], []
    r = 1
    for _ in range(nblocks):
        d, tag, typ, n = map(int, el[r].split())
        r += 1
        for k in range(n):
            v = list(map(int, el[r + k].split()))
            if typ == 3:
                quads.append((d, tag, v[1:5]))
            elif typ == 1:
                lines.append((d, tag, v[1:3]))
            elif typ not in (15,):
                raise NotImplementedError(f"element type {typ} (only points, lines and quadrangles)")
        r += n
    if not quads:
        raise NotImplementedError("no quadrangles")
    # logical coordinates by propagation from the first quadrangle
    offs = ((0, 0), (1, 0), (1, 1), (0, 1))
    by_node = collections.defaultdict(list)
    for qi, (_, _, v) in enumerate(quads):
        for k, n in enumerate(v):
            by_node[n].append((qi, k))
    ij: dict[int, tuple[int, int]] = {}
    q0 = quads[0][2]
    for k, n in enumerate(q0):
        ij[n] = offs[k]
    done = set()
    todo = collections.deque([0])
    while todo:
        qi = todo.popleft()
        if qi in done:
            continue
        v = quads[qi][2]
        base = None
        for k, n in enumerate(v):
            if n in ij:
                base = (ij[n][0] - offs[k][0], ij[n][1] - offs[k][1])
                break
        if base is None:
            continue
        done.add(qi)
        for k, n in enumerate(v):
            want = (base[0] + offs[k][0], base[1] + offs[k][1])
            if ij.setdefault(n, want) != want:
                raise NotImplementedError("not a logically structured quadrangle grid")
            for qj, _ in by_node[n]:
                if qj not in done:
                    todo.append(qj)
    if len(done) != len(quads):
        raise NotImplementedError("quadrangles not connected")
    i0 = min(a for a, _ in ij.values())
    j0 = min(b for _, b in ij.values())
    ij = {n: (a - i0, b - j0) for n, (a, b) in ij.items()}
    nx = max(a for a, _ in ij.values())
    ny = max(b for _, b in ij.values())
    if nx * ny != len(quads) or len(ij) != (nx + 1) * (ny + 1):
        raise NotImplementedError("not a full rectangle of quadrangles")
    xyz = np.zeros(((nx + 1) * (ny + 1), 3))
    node_tags = np.zeros((nx + 1) * (ny + 1), dtype=np.int64)
    for n, (a, b) in ij.items():
        xyz[a + (nx + 1) * b] = coords[n]
        node_tags[a + (nx + 1) * b] = n
    groups = [None] * (nx * ny)
    order = np.zeros(nx * ny, dtype=np.int64)
    for qi, (d, tag, v) in enumerate(quads):
        a, b = ij[v[0]]
        c = a + nx * b
        if groups[c] is not None:
            raise NotImplementedError("two quadrangles on one cell")
        phys = ent_phys.get((d, tag), [])
        groups[c] = names.get((2, phys[0]), str(phys[0])) if phys else ""
        order[c] = qi
    # boundary groups -> logical sides
    side_nodes = collections.defaultdict(set)
    for d, tag, v in lines:
        for p in ent_phys.get((d, tag), []):
            side_nodes[names.get((1, p), str(p))].update(v)
    sides = {}
    for name, ns in side_nodes.items():
        ijs = [ij[n] for n in ns if n in ij]
        if ijs and all(a == 0 for a, _ in ijs):
            sides[name] = SIDES["i=0"]
        elif ijs and all(a == nx for a, _ in ijs):
            sides[name] = SIDES["i=nx"]
        elif ijs and all(b == 0 for _, b in ijs):
            sides[name] = SIDES["j=0"]
        elif ijs and all(b == ny for _, b in ijs):
            sides[name] = SIDES["j=ny"]
    lib_node = {int(t): q for q, t in enumerate(node_tags)}
    used = [t for t in file_nodes if t in lib_node]
    pos = {t: q + 1 for q, t in enumerate(used)}
    cells = np.zeros(nx * ny, dtype=np.int64)
    cells[order] = np.arange(nx * ny)
    file_order = {"cells": cells.tolist(), "nodes": [lib_node[t] for t in used],
                  "conn": [[pos[t] for t in v] for _, _, v in quads]}
    return {"nx": nx, "ny": ny, "coords": xyz, "cell_groups": groups, "sides": sides,
            "cell_order": order, "node_tags": node_tags, "file_order": file_order}
