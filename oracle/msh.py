"""gmsh 2.2 ASCII reader -- TEST INFRASTRUCTURE ONLY (restates points.cpp).

Used to rebuild the point cloud behind the reference's sample outputs so the
oracle's operators can be pinned against the statistics the reference wrote.

  read_points_xyz_msh    points.cpp:668-697
  read_points_flag_msh   points.cpp:698-793 (2D branch)
  read_elem_vert_complete_msh  points.cpp:569-646
  calc_vert_nb_cv        points.cpp:648-666 (hanging vertices are deleted too)
  calc_elem_normal_2D    points.cpp:498-567
  calc_vert_normal       points.cpp:354-406
  delete_corner_edge_vertices  points.cpp:323-352
"""
from __future__ import annotations

import numpy as np


def read_msh_2d(path: str):
    with open(path) as f:
        tok = f.read().split("\n")
    i = tok.index("$Nodes")
    nv = int(tok[i + 1])
    xyz = np.array([[float(t) for t in tok[i + 2 + k].split()[1:3]] for k in range(nv)])
    j = tok.index("$Elements")
    ne = int(tok[j + 1])
    boundary = np.zeros(nv, bool)
    corner = np.zeros(nv, bool)
    elem_vert, elem_bnd = [], []
    for k in range(ne):
        f_ = [int(t) for t in tok[j + 2 + k].split()]
        typ, ntag = f_[1], f_[2]
        nodes = [v - 1 for v in f_[3 + ntag:]]
        if typ == 15:
            corner[nodes[0]] = True
        elif typ == 1:
            boundary[nodes] = True
            elem_vert.append(nodes[:2])
            elem_bnd.append(True)
        elif typ == 2:
            elem_vert.append(nodes[:3])
            elem_bnd.append(False)
        else:
            raise ValueError(f"unsupported element type {typ}")
    vert_nb = [[] for _ in range(nv)]
    for e, vs in enumerate(elem_vert):
        for v in vs:
            vert_nb[v].append(e)
    for v in range(nv):
        if not vert_nb[v]:
            corner[v] = True
    elem_normal = np.zeros((len(elem_vert), 2))
    for e, vs in enumerate(elem_vert):
        if not elem_bnd[e]:
            continue
        iv0, iv1 = vs
        nrm = np.array([xyz[iv1, 1] - xyz[iv0, 1], -(xyz[iv1, 0] - xyz[iv0, 0])])
        inner = next((c for c in vert_nb[iv0] if not elem_bnd[c]), -1)
        if inner < 0:
            raise ValueError("boundary element without an interior neighbour")
        cen = xyz[elem_vert[inner]].sum(0) / len(elem_vert[inner])
        direction = xyz[iv1] - cen
        if direction @ nrm < 0:
            nrm = -nrm
        elem_normal[e] = nrm / np.sqrt(nrm @ nrm)
    normal = np.zeros((nv, 2))
    for v in range(nv):
        if boundary[v]:
            cs = [c for c in vert_nb[v] if elem_bnd[c]]
            s = sum(elem_normal[c] for c in cs) / len(cs)
            normal[v] = s / np.sqrt(s @ s)
    keep = ~corner
    return xyz[keep], boundary[keep], normal[keep]


def charac_dx(xyz: np.ndarray, nb_col: np.ndarray):
    """cloud.cpp:281-313: per node, distance to the nearest other stencil member;
    returns (max, min, avg)."""
    d = np.sqrt(((xyz[nb_col] - xyz[:, None, :]) ** 2).sum(-1))
    d[nb_col == np.arange(len(xyz))[:, None]] = np.inf
    local = d.min(1)
    return float(local.max()), float(local.min()), float(local.mean())
