"""Post-processing and I/O of postprocessing_functions.cpp for GPU clouds.

  calc_max_l1_error                   general_functions.cpp:940-1032
  calc_navier_stokes_residuals_2D     postprocessing_functions.cpp:182-208 (operators on the GPU)
  write_navier_stokes_residuals_2D    :370-401
  calc_navier_stokes_errors_2D / write_navier_stokes_errors_2D   :154-180, :336-368
  write_iteration_details             :52-72
  write_tecplot_steady_variables      :765-805
  write_tecplot_temporal_variables_header / write_tecplot_temporal_variables   :403-416, :476-509
  read_restart_tecplot_file           :597-682 (nearest node by the GPU probe kNN)
  write_csv_xyz / write_csv_temporal_data_init / write_csv_temporal_data      :855-893

The reference writes the mesh's original vertices with their triangles /
tetrahedra (points.xyz_original, elem_vert_original) and the value of the
nearest renumbered node (iv_original_nearest_vert).  Point clouds built here
carry no elements: the input order plays the original one (POINTS.order maps it
to the current numbering), and `elements` may be passed when a mesh exists;
without it the zone lists ELEMENTS=0.
"""
from __future__ import annotations

import re

import numpy as np

from . import capi
from .capi import check, ptr


def _max_l1(d):
    """The reference's pair: the maximum from 0 by `max_err < |d|`, which skips NaN,
    and the sum over the count, which carries NaN and is 0/0 = NaN for no entries."""
    finite = d[~np.isnan(d)]
    mx = float(finite.max(initial=0.0))
    with np.errstate(invalid="ignore", divide="ignore"):
        l1 = float(np.float64(d.sum()) / np.float64(d.size))
    return mx, l1


def calc_max_l1_error(a1, a2, boundary_flag=None):
    """(max |a1 - a2|, mean |a1 - a2|); with boundary_flag also the boundary and
    internal pairs: (max_b, l1_b, max_i, l1_i).  NaN differences do not enter the
    maxima and make the means NaN, and an empty part has mean NaN, as in the
    reference's loops."""
    d = np.abs(np.asarray(a1, np.float64) - np.asarray(a2, np.float64))
    if boundary_flag is None:
        return _max_l1(d)
    b = np.asarray(boundary_flag, bool)
    return _max_l1(d[b]) + _max_l1(d[~b])


def calc_navier_stokes_residuals_2D(points, cloud, parameters, u, v, p):
    """Continuity and momentum residuals of a 2D field with the cloud's operators (GPU
    SpMVs), as (max, mean) pairs internal / boundary / overall for each equation."""
    if parameters.rho < 0 or parameters.mu < 0:
        raise capi.MemphysError(capi.MP_BAD_ARG, "calc_navier_stokes_residuals_2D: set rho and mu")
    gx = cloud.operator(capi.MP_GRAD_X)
    gy = cloud.operator(capi.MP_GRAD_Y)
    lap = cloud.operator(capi.MP_LAPLACIAN)
    u, v = np.ascontiguousarray(u, np.float64), np.ascontiguousarray(v, np.float64)
    ph = np.ascontiguousarray(np.asarray(p, np.float64)[: points.nv])
    rho, mu = parameters.rho, parameters.mu
    res = {
        "continuity": gx @ u + gy @ v,
        "x_momentum": u * (gx @ u) + v * (gy @ u) - (mu * (lap @ u) / rho) + (gx @ ph) / rho,
        "y_momentum": u * (gx @ v) + v * (gy @ v) - (mu * (lap @ v) / rho) + (gy @ ph) / rho,
    }
    out = {}
    zero = np.zeros(points.nv)
    for k, r in res.items():
        mb, lb, mi, li = calc_max_l1_error(zero, r, points.boundary_flag)
        m, l1 = calc_max_l1_error(zero, r)
        out[k] = {"internal": (mi, li), "boundary": (mb, lb), "overall": (m, l1)}
    return out


_ERR_HEAD = ",max_internal,avg_internal,max_boundary,avg_boundary,max_overall,avg_overall\n"


def _split_row(name, a1, a2, boundary_flag):
    """name, then (max, mean) internal, boundary, overall; the split covers the first
    nv entries (the reference indexes the flags past nv for a bordered pressure)."""
    nv = len(boundary_flag)
    mb, lb, mi, li = calc_max_l1_error(np.asarray(a1)[:nv], np.asarray(a2)[:nv], boundary_flag)
    m, l1 = calc_max_l1_error(a1, a2)
    return name, (mi, li, mb, lb, m, l1)


def _row_text(name, vals):
    return name + "".join(f",{v:.16g}" for v in vals) + "\n"


def _residual_rows(points, cloud, parameters, u, v, p):
    gx = cloud.operator(capi.MP_GRAD_X)
    gy = cloud.operator(capi.MP_GRAD_Y)
    lap = cloud.operator(capi.MP_LAPLACIAN)
    u, v = np.asarray(u, np.float64), np.asarray(v, np.float64)
    ph = np.asarray(p, np.float64)[: points.nv]
    rho, mu = parameters.rho, parameters.mu
    zero = np.zeros(points.nv)
    return [
        _split_row("continuity", zero, gx @ u + gy @ v, points.boundary_flag),
        _split_row("X-mom", zero, u * (gx @ u) + v * (gy @ u) - (mu * (lap @ u) / rho)
                   + (gx @ ph) / rho, points.boundary_flag),
        _split_row("Y-mom", zero, u * (gx @ v) + v * (gy @ v) - (mu * (lap @ v) / rho)
                   + (gy @ ph) / rho, points.boundary_flag),
    ]


def write_navier_stokes_residuals_2D(prefix, suffix, points, cloud, parameters, u, v, p):
    """<prefix><suffix>: the residual table of :370-401 (GPU operators)."""
    if parameters.rho < 0 or parameters.mu < 0:
        raise capi.MemphysError(capi.MP_BAD_ARG, "write_navier_stokes_residuals_2D: set rho and mu")
    path = prefix + suffix
    with open(path, "w") as f:
        f.write("Numerical,Residuals,wrt,Given,solution\n" + _ERR_HEAD)
        for name, vals in _residual_rows(points, cloud, parameters, u, v, p):
            f.write(_row_text(name, vals))
    return path


def calc_navier_stokes_errors_2D(points, cloud, u_ana, v_ana, p_ana, u_num, v_num, p_num):
    """Continuity residual and the errors of u, v, p against an analytic solution
    (:154-180), as {name: (max_internal, avg_internal, max_boundary, avg_boundary,
    max_overall, avg_overall)}.  The pressure is shifted to the analytic level at
    node 0 first; the inputs are not modified (the reference shifts p_num in place)."""
    gx = cloud.operator(capi.MP_GRAD_X)
    gy = cloud.operator(capi.MP_GRAD_Y)
    zero = np.zeros(points.nv)
    pn = np.asarray(p_num, np.float64).copy()
    pa = np.asarray(p_ana, np.float64).copy()
    pn = pn - (pn[0] - pa[0])
    if len(pa) == points.nv + 1:
        pa[points.nv] = 0.0
        pn[points.nv] = 0.0
    rows = [
        _split_row("continuity", zero, gx @ np.asarray(u_num, np.float64)
                   + gy @ np.asarray(v_num, np.float64), points.boundary_flag),
        _split_row("U X-vel", u_ana, u_num, points.boundary_flag),
        _split_row("V Y-vel", v_ana, v_num, points.boundary_flag),
        _split_row("Pressure", pa, pn, points.boundary_flag),
    ]
    return dict(rows)


def write_navier_stokes_errors_2D(prefix, points, cloud, u_ana, v_ana, p_ana, u_num, v_num,
                                  p_num):
    """<prefix>_navier_stokes_errors.csv: the table of :336-368."""
    path = prefix + "_navier_stokes_errors.csv"
    errs = calc_navier_stokes_errors_2D(points, cloud, u_ana, v_ana, p_ana, u_num, v_num, p_num)
    with open(path, "w") as f:
        f.write("Errors,wrt,Analytical,solution\n" + _ERR_HEAD)
        for name, vals in errs.items():
            f.write(_row_text(name, vals))
    return path


def write_iteration_details(prefix, n_iter_actual, rel_res_log, abs_res_log, regul_alpha_log=()):
    """<prefix>_iteration_details.csv (:52-72): one row per logged solve."""
    path = prefix + "_iteration_details.csv"
    with open(path, "w") as f:
        if len(regul_alpha_log) == 0:
            f.write("it,n_iter_actual,rel_res_log,abs_res_log\n")
            for it, (n, r, a) in enumerate(zip(n_iter_actual, rel_res_log, abs_res_log)):
                f.write(f"{it},{int(n)},{r:.16g},{a:.16g}\n")
        else:
            f.write("it,n_iter_actual,rel_res_log,abs_res_log,regul_alpha_log\n")
            for it, (n, r, a, g) in enumerate(zip(n_iter_actual, rel_res_log, abs_res_log,
                                                   regul_alpha_log)):
                f.write(f"{it},{int(n)},{r:.16g},{a:.16g},{g:.16g}\n")
    return path


def _original(points):
    """Coordinates in the input order and, for each, the current node holding it."""
    if points.order is None:
        return points.xyz, np.arange(points.nv)
    return points.xyz[points.order], np.asarray(points.order)


def _variables_line(dim, names):
    head = 'VARIABLES="x", "y"' if dim == 2 else 'VARIABLES="x", "y", "z"'
    return head + "".join(f', "{n}"' for n in names) + "\n"


def _zone(t, nv, elements, dim):
    ncv = 0 if elements is None else sum(1 for e in elements if len(e) == dim + 1)
    kind = "FETRIANGLE" if dim == 2 else "FETETRAHEDRON"
    return f'ZONE T="{t:.16g}"  DATAPACKING=POINT, NODES={nv}, ELEMENTS={ncv}, ZONETYPE={kind}\n'


def _rows(points, fields, elements):
    xyz, cur = _original(points)
    lines = []
    for i in range(points.nv):
        vals = [f"{x:.16g} " for x in xyz[i]] + [f"{np.asarray(f)[cur[i]]:.16g} " for f in fields]
        lines.append("".join(vals) + "\n")
    if elements is not None:
        for e in elements:
            if len(e) == points.dim + 1:
                lines.append("".join(f"{int(k) + 1} " for k in e) + "\n")
    return lines


def write_tecplot_steady_variables(prefix, points, names, fields, elements=None):
    """<prefix>_tecplot.plt: one zone at T = 1 with x, y[, z] and the fields."""
    path = prefix + "_tecplot.plt"
    with open(path, "w") as f:
        f.write(_variables_line(points.dim, names))
        f.write(_zone(1.0, points.nv, elements, points.dim))
        f.writelines(_rows(points, fields, elements))
    return path


def write_tecplot_temporal_variables_header(prefix, dim, names):
    path = prefix + "_tecplot_temporal.plt"
    with open(path, "w") as f:
        f.write(_variables_line(dim, names))
    return path


def write_tecplot_temporal_variables(prefix, points, dt, names, fields, it, elements=None):
    """Appends one zone at T = it * dt to <prefix>_tecplot_temporal.plt."""
    path = prefix + "_tecplot_temporal.plt"
    with open(path, "a") as f:
        f.write(_zone(it * dt, points.nv, elements, points.dim))
        f.writelines(_rows(points, fields, elements))
    return path


def read_restart_tecplot_file(points, filename, names):
    """The named variables of the first zone of a Tecplot file, each node taking the
    value of the nearest point of the file (read_restart_tecplot_file :597-682)."""
    with open(filename) as f:
        first = f.readline()
        second = f.readline()
        words = first.split()
        idx = []
        for n in names:
            # the reference looks for '"name",' only, which misses the last variable
            hits = [k for k, w in enumerate(words) if w in (f'"{n}",', f'"{n}"')]
            if not hits:
                raise capi.MemphysError(capi.MP_BAD_ARG, f"unable to find variable {n} in the "
                                                         f"first line of {filename}")
            idx.append(hits[0] - points.dim)  # past "X", "Y"[, "Z"]
        m = re.search(r"NODES\D*(\d+)", second)
        if not m:
            raise capi.MemphysError(capi.MP_BAD_ARG, f"no NODES in the second line of {filename}")
        nvt = int(m.group(1))
        nvar = len(words) - points.dim
        data = np.loadtxt(f, max_rows=nvt, ndmin=2)
    dim = points.dim
    if data.shape != (nvt, dim + nvar):
        raise capi.MemphysError(capi.MP_BAD_ARG, f"{filename}: expected {nvt} rows of "
                                                 f"{dim + nvar} values")
    src = np.ascontiguousarray(data[:, :dim])
    near = np.zeros((points.nv, 1), np.int32)
    check(capi.lib().mp_knn_probe(ptr(src), nvt, dim, ptr(np.ascontiguousarray(points.xyz)),
                                  points.nv, 1, ptr(near), None), "mp_knn_probe")
    return [data[near[:, 0], dim + k].copy() for k in idx]


def write_csv_xyz(xyz, dim, file_name):
    xyz = np.asarray(xyz, np.float64).reshape(-1, dim)
    with open(file_name, "w") as f:
        f.write("no,x,y\n" if dim == 2 else "no,x,y,z\n")
        for i, p in enumerate(xyz):
            f.write(f"{i}," + ",".join(f"{c:.16g}" for c in p) + "\n")


def write_csv_temporal_data_init(size, file_name):
    with open(file_name, "w") as f:
        f.write("time(s)" + "".join(f",{i}" for i in range(size)) + "\n")


def write_csv_temporal_data(data, time, file_name):
    with open(file_name, "a") as f:
        f.write(f"{time:.16g}" + "".join(f",{x:.16g}" for x in np.asarray(data, np.float64)) + "\n")
