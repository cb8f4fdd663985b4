"""SU2 mesh reader of the oracle (test infrastructure, not product code).

CPU restatement of Mesh2D::LoadSU2MeshFromFile (code/src/mesh2d.cpp:68-259)
and of the [mesh] SU2BC table (mesh2d.cpp:21-56), returning the arrays the
oracle and the reference harness take:

  xy             (nNodes, 2) node coordinates, nodes sorted by their file id
                 (mesh2d.cpp:80-102)
  node_boundary  1 for nodes of any marker element (:120-134)
  tri            (nCells, 3) node indices of each triangle, file order
                 (:161-195); quadrangles are refused
  cell_bc        per cell: 0 interior, 1 dirichlet, 2 noslip, 3 swwall. A
                 triangle with exactly two boundary nodes is a boundary cell
                 (triangle.cpp:10-16); its type comes from the loop of
                 :199-214 -- for each of its nodes, each marker, each marker
                 element whose first or second node is that node, the
                 marker's type, the last match winning.

The mesh2d.cpp file itself needs VTK and is not compiled by the harness; this
reader is pinned by the tests against hand-derived cases and against the
product's own reader, and the harness takes its arrays.
"""
from __future__ import annotations

import re

import numpy as np

BC_CODES = {"dirichlet": 1, "noslip": 2, "swwall": 3}


def _trailing(line: str) -> int:
    """Mesh2D::GetTrailingNumber (mesh2d.cpp:261-263): the number from the first digit on."""
    m = re.search(r"\d+", line)
    if m is None:
        raise ValueError(f"no number in {line!r}")
    return int(m.group(0))


def bc_table(su2bc) -> dict:
    """[mesh] SU2BC = [[tag, type], ...] -> {tag: code} (mesh2d.cpp:30-52)."""
    out = {}
    for tag, kind in su2bc:
        if kind not in BC_CODES:
            raise ValueError(f"boundary condition {kind!r} on {tag!r} is not supported")
        out[tag] = BC_CODES[kind]
    return out


def read_su2(path: str, bcs: dict) -> dict:
    lines = [l.rstrip("\r\n") for l in open(path)]

    def find(key):
        for i, l in enumerate(lines):
            if key in l:
                return i
        raise ValueError(f"{key} not found in {path}")

    at = find("NPOIN")
    n_pts = _trailing(lines[at])
    pts = []
    for i in range(n_pts):
        f = lines[at + 1 + i].split()
        pts.append((int(f[2]) if len(f) > 2 else i, float(f[0]), float(f[1])))
    pts.sort(key=lambda p: p[0])
    index = {p[0]: n for n, p in enumerate(pts)}
    xy = np.array([[p[1], p[2]] for p in pts], dtype=np.float64)

    node_bnd = np.zeros(n_pts, dtype=np.int32)
    markers = []    # (code, [(node0, node1), ...]) in file order
    at = find("NMARK")
    k = at + 1
    for _ in range(_trailing(lines[at])):
        tag, elems = None, []
        for _part in range(2):
            l = lines[k]
            k += 1
            if "MARKER_TAG" in l:
                tag = "".join(l.split("=", 1)[1].split())
            elif "MARKER_ELEMS" in l:
                for _e in range(_trailing(l)):
                    f = lines[k].split()
                    k += 1
                    a, b = index[int(f[1])], index[int(f[2])]
                    node_bnd[a] = node_bnd[b] = 1
                    elems.append((a, b))
            else:
                raise ValueError(f"unexpected line {l!r}")
        if tag not in bcs:
            raise ValueError(f"no SU2BC entry for marker {tag!r}")
        markers.append((bcs[tag], elems))

    at = find("NELEM")
    n_el = _trailing(lines[at])
    tri = np.zeros((n_el, 3), dtype=np.int32)
    for c in range(n_el):
        f = lines[at + 1 + c].split()
        if int(f[0]) != 5:
            raise ValueError("only triangles (type 5) are supported")
        tri[c] = [index[int(v)] for v in f[1:4]]

    cell_bc = np.zeros(n_el, dtype=np.int32)
    for c in range(n_el):
        if int(node_bnd[tri[c]].sum()) != 2:
            continue
        code = 1
        for nid in tri[c]:
            for mcode, elems in markers:
                for a, b in elems:
                    if a == nid or b == nid:
                        code = mcode
        cell_bc[c] = code
    return dict(xy=xy, node_boundary=node_bnd, tri=tri, cell_bc=cell_bc)
