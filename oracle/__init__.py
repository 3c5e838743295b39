"""CPU oracle for the MeMPhyS hot path -- TEST INFRASTRUCTURE ONLY.

This package is what the CUDA product path is compared against in the tests, and
the CPU baseline that ``bench.py`` times beside the GPU.  It is imported only by
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s cpu-baseline leg;
nothing under ``memphys_b200/`` imports it.

The numerics live in ``memphys_oracle.c`` (a restatement of the reference's
``coefficient_computations.cpp``, ``cloud.cpp``, ``solver.cpp`` and
``fractional_step_1.cpp``); this module binds it with ctypes.  ``msh.py``
restates the gmsh reader of ``points.cpp`` for the sample-output pins.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import scipy.sparse as sp

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libmemphys_oracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_bp = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    """Compile the oracle shared library with the committed Makefile."""
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
        os.path.join(_HERE, "memphys_oracle.c")
    ):
        subprocess.run(["make", "-s", "-C", _HERE, "libmemphys_oracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        L.mo_num_poly_terms.argtypes = [C.c_int, C.c_int]
        L.mo_cloud_size.argtypes = [C.c_int, C.c_int, C.c_double]
        L.mo_poly_exponents.argtypes = [C.c_int, C.c_int, _ip]
        L.mo_poly_exponents.restype = None
        L.mo_stencil_single.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_int, _ip, _dp,
                                        C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.mo_cloud_weights.argtypes = [_dp, C.c_int, C.c_int, _ip, _ip, C.c_int, C.c_int,
                                       _dp, _dp, C.c_void_p, _dp, C.c_void_p, C.c_void_p]
        L.mo_batched_weights.argtypes = [C.c_int, _ip, _lp, _dp, C.c_int, C.c_int, C.c_int,
                                         _dp, C.c_void_p]
        L.mo_knn_stencils.argtypes = [_dp, _bp, C.c_int, C.c_int, C.c_int, _ip]
        L.mo_spmv_csr.argtypes = [C.c_int, _ip, _ip, _dp, _dp, _dp]
        L.mo_spmv_csr.restype = None
        L.mo_ppe_assemble.argtypes = [C.c_int, C.c_int, C.c_int, _ip, _dp, _dp, C.c_void_p, _dp,
                                      _bp, _bp, _dp, C.c_double, C.c_double, C.c_double, C.c_int,
                                      _ip, _ip, _dp]
        L.mo_ilut_create.argtypes = [C.c_int, _ip, _ip, _dp, C.c_double, C.c_int]
        L.mo_ilut_create.restype = C.c_void_p
        L.mo_ilut_destroy.argtypes = [C.c_void_p]
        L.mo_ilut_destroy.restype = None
        L.mo_ilut_apply.argtypes = [C.c_void_p, _dp, _dp]
        L.mo_ilut_apply.restype = None
        L.mo_ilut_nnz.argtypes = [C.c_void_p]
        L.mo_ilut_nnz.restype = C.c_longlong
        L.mo_bicgstab.argtypes = [C.c_int, _ip, _ip, _dp, C.c_void_p, _dp, _dp, C.c_double,
                                  C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.mo_fs1_create.argtypes = [C.c_int, C.c_int, C.c_int, _ip, _dp, _dp, C.c_void_p, _dp,
                                    _bp, _dp, _bp, _bp, C.c_void_p, _bp, C.c_double, C.c_double,
                                    C.c_double, C.c_int, C.c_double, C.c_int, C.c_double, C.c_int,
                                    C.c_int]
        L.mo_fs1_create.restype = C.c_void_p
        L.mo_fs1_system_size.argtypes = [C.c_void_p]
        L.mo_fs1_step.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), _dp, C.c_int,
                                  C.POINTER(C.c_double)]
        L.mo_fs1_destroy.argtypes = [C.c_void_p]
        L.mo_fs1_destroy.restype = None
        L.mo_set_threads.argtypes = [C.c_int]
        L.mo_set_threads.restype = C.c_int
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------- parameters
def set_threads(n: int) -> int:
    """Threads of the oracle's row-parallel loops (OpenMP); returns the previous
    count.  Dot products and ILUT solves stay serial, so results do not change."""
    return lib().mo_set_threads(int(n))


def num_poly_terms(dim: int, poly_deg: int) -> int:
    """parameters.cpp:122-130."""
    return lib().mo_num_poly_terms(dim, poly_deg)


def cloud_size(dim: int, poly_deg: int, multiplier: float) -> int:
    """parameters.cpp:128."""
    return lib().mo_cloud_size(dim, poly_deg, multiplier)


def poly_exponents(dim: int, poly_deg: int) -> np.ndarray:
    """parameters.cpp:217-267, shape (m, dim)."""
    m = num_poly_terms(dim, poly_deg)
    e = np.zeros(m * dim, np.int32)
    lib().mo_poly_exponents(dim, poly_deg, e)
    return e.reshape(m, dim)


# ---------------------------------------------------------------- stencils
def knn_stencils(xyz: np.ndarray, boundary: np.ndarray, n: int) -> np.ndarray:
    """cloud.cpp:570-648 stencil rule; returns (nv, n) int32, row i = stencil of node i."""
    xyz = np.ascontiguousarray(xyz, np.float64)
    nv, dim = xyz.shape
    out = np.zeros(nv * n, np.int32)
    fail = lib().mo_knn_stencils(xyz.ravel(), np.ascontiguousarray(boundary, np.uint8), nv, dim, n, out)
    if fail:
        raise RuntimeError(f"oracle kNN: {fail} nodes without enough neighbours")
    return out.reshape(nv, n)


def stencil_single(vert: np.ndarray, phs: int, poly_deg: int):
    """coefficient_computations.cpp:294-328 for one stencil (row 0 = centre).

    Returns (w[(dim+1), n], cond_estimate, cond_exact)."""
    vert = np.ascontiguousarray(vert, np.float64)
    n, dim = vert.shape
    e = poly_exponents(dim, poly_deg)
    m = e.shape[0]
    w = np.zeros((dim + 1) * n)
    ce, cx = C.c_double(), C.c_double()
    info = lib().mo_stencil_single(vert.ravel(), n, dim, phs, m, e.ravel().copy(), w,
                                   C.byref(ce), C.byref(cx))
    if info:
        raise FloatingPointError(f"singular stencil (zero pivot {info - 1})")
    return w.reshape(dim + 1, n), ce.value, cx.value


def cloud_weights(xyz, nb_col, phs=3, poly_deg=3, cond=True):
    """cloud.cpp:207-279.  nb_col: (nv, n) stencils.  Returns dict of CSR-aligned
    (nv, n) arrays gx, gy, [gz], lap and per-node cond_est / cond_exact."""
    xyz = np.ascontiguousarray(xyz, np.float64)
    dim = xyz.shape[1]
    nb_col = np.ascontiguousarray(nb_col, np.int32)
    nv, n = nb_col.shape  # stencils to solve (may be a subset of the cloud's nodes)
    if nb_col.size and (nb_col.min() < 0 or nb_col.max() >= xyz.shape[0]):
        raise IndexError("stencil index outside the cloud")
    rp = (np.arange(nv + 1, dtype=np.int32) * n)
    gx, gy, lap = (np.zeros(nv * n) for _ in range(3))
    gz = np.zeros(nv * n) if dim == 3 else None
    ce = np.zeros(nv) if cond else None
    cx = np.zeros(nv) if cond else None
    bad = lib().mo_cloud_weights(xyz.ravel(), nv, dim, rp, nb_col.ravel(), phs, poly_deg, gx, gy,
                                 _ptr(gz), lap, _ptr(ce), _ptr(cx))
    out = {"gx": gx.reshape(nv, n), "gy": gy.reshape(nv, n), "lap": lap.reshape(nv, n),
           "singular": bad}
    if gz is not None:
        out["gz"] = gz.reshape(nv, n)
    if cond:
        out["cond_est"] = ce
        out["cond_exact"] = cx
    return out


def batched_weights(sizes, offsets, pts, dim, phs=3, poly_deg=3, cond=False):
    """Independent uneven stencils (batched-solve workload); w laid out per system
    as (dim+1) x n_i at (dim+1)*offsets[i]."""
    sizes = np.ascontiguousarray(sizes, np.int32)
    offsets = np.ascontiguousarray(offsets, np.int64)
    pts = np.ascontiguousarray(pts, np.float64).ravel()
    total = int(offsets[-1] + sizes[-1]) if len(sizes) else 0
    w = np.zeros((dim + 1) * total)
    cx = np.zeros(len(sizes)) if cond else None
    bad = lib().mo_batched_weights(len(sizes), sizes, offsets, pts, dim, phs, poly_deg, w, _ptr(cx))
    return w, cx, bad


# ---------------------------------------------------------------- operators
def interp_matrix(xyz: np.ndarray, probe: np.ndarray, n: int, phs: int = 3, poly_deg: int = 3):
    """calc_interp_matrix (coefficient_computations.cpp:456-518) in numpy: each probe's n
    nearest nodes (calc_cloud_points_slow for probes, :373-428; here ordered by distance,
    ties by index), shifting_scaling of the stencil with the probe (:4-31), the saddle
    matrix of :70-106 and the right-hand side of :430-454, solved by LAPACK.
    Returns cols (np x n) and weights (np x n)."""
    xyz = np.asarray(xyz, np.float64)
    probe = np.asarray(probe, np.float64)
    dim = xyz.shape[1]
    e = poly_exponents(dim, poly_deg)
    m = e.shape[0]
    cols = np.zeros((len(probe), n), np.int32)
    wts = np.zeros((len(probe), n))
    idx = np.arange(len(xyz))
    for q, p in enumerate(probe):
        d2 = ((xyz - p) ** 2).sum(1)
        nb = np.lexsort((idx, d2))[:n]
        v = xyz[nb].copy()
        lo, hi = v.min(0), v.max(0)
        sc = hi - lo
        v = (v - lo) / sc
        xp = (p - lo) / sc
        r2 = ((v[:, None, :] - v[None, :, :]) ** 2).sum(2)
        A = np.zeros((n + m, n + m))
        A[:n, :n] = r2 ** (phs / 2.0)
        np.fill_diagonal(A[:n, :n], 0.0)
        P = np.prod(v[:, None, :] ** e[None, :, :], axis=2)
        A[:n, n:] = P
        A[n:, :n] = P.T
        rhs = np.zeros(n + m)
        rhs[:n] = ((v - xp) ** 2).sum(1) ** (phs / 2.0)
        rhs[n:] = np.prod(xp[None, :] ** e, axis=1)
        cols[q] = nb
        wts[q] = np.linalg.solve(A, rhs)[:n]
    return cols, wts


def rcm_order(nb_col: np.ndarray) -> np.ndarray:
    """reverse_cuthill_mckee_ordering (general_functions.cpp:806-879) on the stencil
    graph, as CLOUD::re_order_points_reverse_cuthill_mckee builds it (cloud.cpp:315-335):
    adjacency of node i = its stencil row; breadth-first from the first node of least
    degree, each node's unvisited neighbours appended sorted by (degree, index); then
    order[i] = nv - 1 - position.  Pure Python: small clouds only."""
    nb = np.asarray(nb_col)
    nv = nb.shape[0]
    degree = [len(row) for row in nb]
    visited = [False] * nv
    start = min(range(nv), key=lambda i: (degree[i], i))
    numbering = [start]
    visited[start] = True
    index = 0
    while len(numbering) < nv:
        if index == len(numbering):  # not reached from the start (the reference reads past)
            nxt = min((i for i in range(nv) if not visited[i]), key=lambda i: (degree[i], i))
            visited[nxt] = True
            numbering.append(nxt)
        v = numbering[index]
        index += 1
        fresh = []
        for w in nb[v]:
            w = int(w)
            if not visited[w]:
                visited[w] = True
                fresh.append((degree[w], w))
        numbering.extend(w for _, w in sorted(fresh))
    order = np.empty(nv, np.int32)
    order[np.asarray(numbering)] = np.arange(nv, dtype=np.int32)
    return (nv - 1 - order).astype(np.int32)


def ell_to_csr(nb_col: np.ndarray):
    nv, n = nb_col.shape
    return np.arange(nv + 1, dtype=np.int32) * n, np.ascontiguousarray(nb_col.ravel(), np.int32)


def spmv(rp, ci, val, x):
    y = np.zeros(len(rp) - 1)
    lib().mo_spmv_csr(len(rp) - 1, rp, ci, np.ascontiguousarray(val, np.float64).ravel(),
                      np.ascontiguousarray(x, np.float64), y)
    return y


def ppe_assemble(nb_col, w, boundary, dirichlet, normal, unsteady=0.0, conv=0.0, diff=1.0,
                 bordered=None):
    """solver.cpp:165-214.  Returns CSR (rp, ci, val) and the system size."""
    nb_col = np.ascontiguousarray(nb_col, np.int32)
    nv, n = nb_col.shape
    dim = normal.shape[1]
    bflag = np.ascontiguousarray(boundary, np.uint8)
    dflag = np.ascontiguousarray(dirichlet, np.uint8)
    if bordered is None:  # solver.cpp:29-38
        bordered = not bool(np.any(bflag & dflag))
    cap = nv * n + 2 * nv + 1
    rp = np.zeros(nv + 2, np.int32)
    ci = np.zeros(cap, np.int32)
    val = np.zeros(cap)
    gz = w.get("gz")
    ns = lib().mo_ppe_assemble(nv, dim, n, nb_col.ravel(), w["gx"].ravel(), w["gy"].ravel(),
                               _ptr(np.ascontiguousarray(gz.ravel()) if gz is not None else None),
                               w["lap"].ravel(), bflag, dflag,
                               np.ascontiguousarray(normal, np.float64).ravel(), unsteady, conv,
                               diff, int(bordered), rp, ci, val)
    rp = rp[: ns + 1].copy()
    return rp, ci[: rp[-1]].copy(), val[: rp[-1]].copy(), ns


def sor_colouring(rp, ci, val, nv):
    """The row colouring of the GPU's multicolour SOR, restated: rows in index order,
    each taking the smallest colour held neither by a member of its own row nor by a
    row that contains it (the graph of the nonzero coefficients made symmetric).
    Returns the colour of every row."""
    rp = np.asarray(rp)
    ci = np.asarray(ci)
    rows = np.repeat(np.arange(nv), np.diff(rp[: nv + 1]))
    cols = ci[: rp[nv]]
    keep = (cols != rows) & (cols < nv) & (np.asarray(val)[: rp[nv]] != 0.0)
    fwd = [[] for _ in range(nv)]
    for i, j in zip(rows[keep].tolist(), cols[keep].tolist()):
        fwd[i].append(j)
        fwd[j].append(i)
    colour = [-1] * nv
    for i in range(nv):
        used = {colour[j] for j in fwd[i] if colour[j] >= 0}
        c = 0
        while c in used:
            c += 1
        colour[i] = c
    return np.asarray(colour)


def sor_sweeps(rp, ci, val, b, x, omega=1.4, sweeps=1, colour=None):
    """SOLVER::SOR's update (solver.cpp:243-281): x_i = omega (b_i - sum_{j != i} a_ij
    x_j) / a_ii + (1 - omega) x_i, rows in index order (colour None, the reference's
    order, pure Python: small systems) or colour by colour (the GPU's order; rows of
    one colour never read one another, so each colour is one vector update)."""
    A = sp.csr_matrix((np.asarray(val), np.asarray(ci), np.asarray(rp)))
    n = A.shape[0]
    d = A.diagonal()
    x = np.array(x, np.float64, copy=True)
    if colour is None:
        for _ in range(sweeps):
            for i in range(n):
                lo, hi = A.indptr[i], A.indptr[i + 1]
                s = b[i] - A.data[lo:hi] @ x[A.indices[lo:hi]] + d[i] * x[i]
                x[i] = omega * s / d[i] + (1.0 - omega) * x[i]
        return x
    groups = [np.nonzero(colour == c)[0] for c in range(int(colour.max()) + 1)]
    blocks = [A[g] for g in groups]
    for _ in range(sweeps):
        for g, Ag in zip(groups, blocks):
            s = b[g] - Ag @ x + d[g] * x[g]
            x[g] = omega * s / d[g] + (1.0 - omega) * x[g]
    return x


class ILUT:
    """Saad ILUT(tau, p) restatement of Eigen::IncompleteLUT (solver.cpp:61-67,156)."""

    def __init__(self, rp, ci, val, droptol=1e-4, fill=100):
        self.n = len(rp) - 1
        self.h = lib().mo_ilut_create(self.n, rp, ci, np.ascontiguousarray(val), droptol, fill)

    def apply(self, b):
        x = np.zeros(self.n)
        lib().mo_ilut_apply(self.h, np.ascontiguousarray(b, np.float64), x)
        return x

    def nnz(self):
        return lib().mo_ilut_nnz(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().mo_ilut_destroy(self.h)
            self.h = None


def bicgstab(rp, ci, val, b, x0=None, tol=1e-8, maxit=1000, precond: ILUT | None = None):
    """solver.cpp:337-350 (Eigen BiCGSTAB).  Returns (x, iters, true_relres, recursive_relres)."""
    n = len(rp) - 1
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64, copy=True)
    rr, rec = C.c_double(), C.c_double()
    it = lib().mo_bicgstab(n, rp, ci, np.ascontiguousarray(val), precond.h if precond else None,
                           np.ascontiguousarray(b, np.float64), x, tol, maxit, C.byref(rr),
                           C.byref(rec))
    return x, it, rr.value, rec.value


class FS1:
    """fractional_step_1.cpp: FRACTIONAL_STEP_1 with SOLVER(eigen_ilu_bicgstab) for p."""

    def __init__(self, cloud, nb_col, w, rho, mu, dt, temporal_order=2, tol=1e-8, maxit=1000,
                 droptol=1e-4, fill=100, use_ilut=True):
        self.keep = []
        nb_col = np.ascontiguousarray(nb_col, np.int32)
        nv, n = nb_col.shape
        dim = cloud.dim
        self.nv, self.dim = nv, dim

        def k(a, dt_=np.float64):
            a = np.ascontiguousarray(a, dt_).ravel()
            self.keep.append(a)
            return a

        gz = k(w["gz"]) if dim == 3 else None
        wdir = k(cloud.w_dirichlet, np.uint8) if dim == 3 else None
        self.h = lib().mo_fs1_create(
            nv, dim, n, k(nb_col, np.int32), k(w["gx"]), k(w["gy"]), _ptr(gz), k(w["lap"]),
            k(cloud.boundary, np.uint8), k(cloud.normal), k(cloud.u_dirichlet, np.uint8),
            k(cloud.v_dirichlet, np.uint8), _ptr(wdir), k(cloud.p_dirichlet, np.uint8), rho, mu,
            dt, temporal_order, tol, maxit, droptol, fill, int(use_ilut))
        self.nsys = lib().mo_fs1_system_size(self.h)

    def step(self, vel, p, it):
        """vel: list of dim float64 arrays (in place); p: float64 array of nsys (in place)."""
        arr = (C.c_void_p * self.dim)(*[v.ctypes.data for v in vel])
        rr = C.c_double()
        iters = lib().mo_fs1_step(self.h, arr, p, it, C.byref(rr))
        return iters, rr.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().mo_fs1_destroy(self.h)
            self.h = None
