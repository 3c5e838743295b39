"""Regenerates the golden fixtures in this folder (run in a tree that has the
reference checkout; the fixtures are committed so tests never need it).

  sample_stats.json   the reference's own sample-output statistics for
                      CAD_Mesh_files/ecc_ratio_0.5_r_i_0.6_n_200.msh, parsed
                      from "Sample outputs/..._simulation_details.csv".
  ecc_cloud.npz       that mesh read by the restated gmsh reader (xyz,
                      boundary flags, normals after corner deletion) plus its
                      stencils from the reference's vendored nanoflann
                      (oracle/_ref/ref_knn, built by `make -C oracle ref`).
  knn_cavity.npz      a 40x40 jittered cavity and its nanoflann stencils.
  lapack_stencils.npz 240 uneven independent PHS systems (2D and 3D) and
                      their weights from scipy's LAPACK dgesv.
  couette_clouds.npz  the concentric annuli CAD_Mesh_files/ecc_ratio_0.0_r_i_0.5_n_100
                      and _n_150.msh read by the restated gmsh reader (xyz,
                      boundary flags, normals), for the concentric-Couette check
                      against the analytic profile of the reference's driver.

usage: python tests/golden/make_golden.py [reference_root] [--only couette]
"""
from __future__ import annotations

import csv
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import msh  # noqa: E402
from memphys_b200 import clouds  # noqa: E402


def ref_knn(xyz, bnd, n):
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_knn")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    with tempfile.TemporaryDirectory() as d:
        fi, fo = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        nv, dim = xyz.shape
        with open(fi, "wb") as f:
            np.array([nv, dim, n], np.int32).tofile(f)
            np.ascontiguousarray(xyz, np.float64).tofile(f)
            np.ascontiguousarray(bnd, np.uint8).tofile(f)
        subprocess.run([exe, fi, fo], check=True)
        return np.fromfile(fo, np.int32).reshape(nv, n)


def sample_stats(ref_root):
    p = os.path.join(ref_root, "MeMPhyS Latest Version", "Sample outputs",
                     "ecc_ratio_0.5_r_i_0.6_n_200_polydeg_3_simulation_details.csv")
    rows = [r for r in csv.reader(open(p)) if r]
    get = {}
    for r in rows:
        key = ",".join(x for x in r[:3] if x and not _isnum(x))
        get[key] = [float(x) for x in r[1:] if _isnum(x)]
    return {
        "source": "Sample outputs/ecc_ratio_0.5_r_i_0.6_n_200_polydeg_3_simulation_details.csv",
        "nv": int(get["No. of,nodes,nv"][0]),
        "nv_boundary": int(get["No. of,nodes,nv_boundary"][0]),
        "dx_max": get["Characteristic,dx_max"][0],
        "dx_min": get["Characteristic,dx_min"][0],
        "dx_avg": get["Characteristic,dx_avg"][0],
        "cond_max": get["RBF_cond_num_max"][0],
        "cond_min": get["RBF_cond_num_min"][0],
        "cond_avg": get["RBF_cond_num_avg"][0],
        "grad_x_eig": get["grad_x_eigval"],
        "grad_y_eig": get["grad_y_eigval"],
        "laplace_eig": get["laplace_eigval"],
        "phs_deg": 3, "poly_deg": 3, "cloud_size": 20,
    }


def _isnum(x):
    try:
        float(x)
        return True
    except ValueError:
        return False


def lapack_stencils(seed=7):
    """Uneven independent systems: offsets in the unit ball scaled by h."""
    from scipy.linalg import lapack
    rng = np.random.Generator(np.random.Philox(seed))
    out = {}
    for dim in (2, 3):
        m = oracle.num_poly_terms(dim, 3)
        e = oracle.poly_exponents(dim, 3)
        sizes = rng.choice([20, 30, 40, 60] if dim == 2 else [40, 50, 60], size=120)
        pts, ws = [], []
        for n in sizes:
            h = rng.uniform(1e-3, 1e-2)
            d = rng.normal(size=(n, dim))
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            d *= rng.uniform(0, 1, size=(n, 1)) ** (1.0 / dim)
            d[0] = 0.0
            x = d * h + rng.uniform(-1, 1, size=dim)
            pts.append(x)
            ws.append(_lapack_weights(x, e, m, lapack))
        out[f"sizes{dim}"] = sizes.astype(np.int32)
        out[f"pts{dim}"] = np.concatenate(pts)
        out[f"w{dim}"] = np.concatenate([w.ravel() for w in ws])
    return out


def _lapack_weights(x, e, m, lapack):
    """coefficient_computations.cpp:70-323 assembled in numpy, solved by dgesv."""
    n, dim = x.shape
    v = x.copy()
    lo, hi = v.min(0), v.max(0)
    sc = hi - lo
    v = (v - lo) / sc
    s = n + m
    A = np.zeros((s, s))
    r2 = ((v[:, None, :] - v[None, :, :]) ** 2).sum(-1)
    A[:n, :n] = r2 ** 1.5
    np.fill_diagonal(A[:n, :n], 0.0)
    P = np.prod(v[:, None, :] ** e[None, :, :], axis=2)
    A[:n, n:] = P
    A[n:, :n] = P.T
    c = v[0]
    rhs = np.zeros((s, dim + 1))
    rc2 = ((v - c) ** 2).sum(-1)
    for k in range(dim):
        rhs[:n, k] = -3.0 * (v[:, k] - c[k]) * rc2 ** 0.5 / sc[k]
        for j in range(m):
            if e[j, k] > 0:
                t = e[j, k] * c[k] ** (e[j, k] - 1.0)
                for q in range(dim):
                    if q != k:
                        t *= c[q] ** e[j, q]
                rhs[n + j, k] = t / sc[k]
    lap = np.zeros(n)
    ok = rc2 > 1e-14
    for k in range(dim):
        dk2 = (v[:, k] - c[k]) ** 2
        lap[ok] += (9.0 * dk2[ok] * rc2[ok] ** -0.5 - 6.0 * dk2[ok] * rc2[ok] ** -0.5
                    + 3.0 * rc2[ok] ** 0.5) / sc[k] ** 2
    rhs[:n, dim] = lap
    for j in range(m):
        acc = 0.0
        for k in range(dim):
            if e[j, k] > 1:
                t = e[j, k] * (e[j, k] - 1.0) * c[k] ** (e[j, k] - 2.0)
                for q in range(dim):
                    if q != k:
                        t *= c[q] ** e[j, q]
                acc += t / sc[k] ** 2
        rhs[n + j, dim] = acc
    lu, piv, sol, info = lapack.dgesv(A, rhs)
    assert info == 0
    return sol[:n].T.copy()  # (dim+1, n)


def couette_clouds(ref_root):
    out = {}
    for n in (100, 150):
        mesh = os.path.join(ref_root, "MeMPhyS Latest Version", "CAD_Mesh_files",
                            f"ecc_ratio_0.0_r_i_0.5_n_{n}.msh")
        xyz, bnd, nrm = msh.read_msh_2d(mesh)
        out[f"xyz_{n}"], out[f"boundary_{n}"], out[f"normal_{n}"] = xyz, bnd, nrm
    np.savez_compressed(os.path.join(HERE, "couette_clouds.npz"), **out)


def main(ref_root="/root/reference", *flags):
    if "--only" in flags:
        what = flags[flags.index("--only") + 1]
        if what == "couette":
            couette_clouds(ref_root)
            print("couette_clouds.npz written to", HERE)
            return
        raise SystemExit(f"unknown fixture {what}")
    couette_clouds(ref_root)
    stats = sample_stats(ref_root)
    with open(os.path.join(HERE, "sample_stats.json"), "w") as f:
        json.dump(stats, f, indent=1)
    mesh = os.path.join(ref_root, "MeMPhyS Latest Version", "CAD_Mesh_files",
                        "ecc_ratio_0.5_r_i_0.6_n_200.msh")
    xyz, bnd, nrm = msh.read_msh_2d(mesh)
    nb = ref_knn(xyz, bnd, 20)
    np.savez_compressed(os.path.join(HERE, "ecc_cloud.npz"), xyz=xyz, boundary=bnd, normal=nrm,
                        nb_col_nanoflann=nb)
    cav = clouds.cavity_2d(40, seed=11)
    nbc = ref_knn(cav.xyz, cav.boundary, 20)
    np.savez_compressed(os.path.join(HERE, "knn_cavity.npz"), xyz=cav.xyz, boundary=cav.boundary,
                        nb_col_nanoflann=nbc)
    np.savez_compressed(os.path.join(HERE, "lapack_stencils.npz"), **lapack_stencils())
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main(*sys.argv[1:])
