"""Host-side mirror of the reference's solver interface over the C ABI.

Same class names, arguments and error behaviour as the reference's
header_files/class.hpp (PARAMETERS :58-94, POINTS :96-140, CLOUD :142-169,
SOLVER :171-217, FRACTIONAL_STEP_1 :246-270); the numerics run in
libmemphys_cuda.so.  Failures raise MemphysError, the counterpart of the
reference's printf + throw bad_exception().
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import capi
from .capi import check, ptr
from .clouds import Cloud

# solver_type strings (parameters.cpp:94-99): the reference's names select the
# closest GPU configuration; the cuda_* names choose one explicitly.
SOLVER_TYPES = {
    "eigen_ilu_bicgstab": dict(precond=capi.MP_PRECOND_AMG, precision=capi.MP_FP64),
    "hypre_ilu_gmres": dict(precond=capi.MP_PRECOND_AMG, precision=capi.MP_FP64),
    "eigen_direct": dict(precond=capi.MP_PRECOND_AMG, precision=capi.MP_FP64),
    "cuda_bicgstab_amg": dict(precond=capi.MP_PRECOND_AMG, precision=capi.MP_FP64),
    "cuda_bicgstab_amg_mixed": dict(precond=capi.MP_PRECOND_AMG, precision=capi.MP_FP32),
    "cuda_bicgstab_amg_mg32": dict(precond=capi.MP_PRECOND_AMG, precision=capi.MP_MG32),
    "cuda_bicgstab_jacobi": dict(precond=capi.MP_PRECOND_JACOBI, precision=capi.MP_FP64),
    "cuda_bicgstab_jacobi_mixed": dict(precond=capi.MP_PRECOND_JACOBI, precision=capi.MP_FP32),
    "cuda_bicgstab": dict(precond=capi.MP_PRECOND_NONE, precision=capi.MP_FP64),
    # SOLVER::SOR (solver.cpp:243-281): SOR sweeps, omega 1.4, unbordered system
    "sor": dict(precond=capi.MP_PRECOND_SOR, precision=capi.MP_FP64),
}


class PARAMETERS:
    """parameters.cpp:27-130,217-267.  Reads the positional parameters CSV, or
    takes the same fields as keyword arguments."""

    FIELDS = ["poly_deg", "phs_deg", "cloud_size_multiplier", "nt", "Courant", "solver_type",
              "steady_tolerance", "solver_tolerance", "euclid_precond_level_hypre", "gmres_kdim",
              "precond_droptol", "n_iter"]

    def __init__(self, parameter_file: str | None = None, dimension: int = 2, **kw):
        vals = dict(poly_deg=3, phs_deg=3, cloud_size_multiplier=2.0, nt=1000, Courant=1.0,
                    solver_type="cuda_bicgstab_amg", steady_tolerance=1e-5, solver_tolerance=1e-8,
                    euclid_precond_level_hypre=50, gmres_kdim=20, precond_droptol=1e-4,
                    n_iter=1000)
        if parameter_file:
            vals.update(self.read_calc_parameters(parameter_file))
        vals.update(kw)
        for k, v in vals.items():
            setattr(self, k, v)
        self.dimension = dimension
        self.rho = -10.0  # class.hpp:74: must be set by the driver
        self.mu = -10.0
        self.dt = None
        self.rel_res_log, self.abs_res_log, self.regul_alpha_log, self.n_iter_actual = [], [], [], []
        self.verify_parameters()
        self.calc_cloud_num_points()
        self.calc_polynomial_term_exponents()

    @classmethod
    def read_calc_parameters(cls, path: str) -> dict:
        """parameters.cpp:42-80: `name,value` lines in fixed order."""
        out = {}
        with open(path) as f:
            lines = [ln.strip() for ln in f if ln.strip()]
        for name, line in zip(cls.FIELDS, lines):
            v = line.split(",", 1)[1].strip()
            if name == "solver_type":
                out[name] = v
            elif name in ("poly_deg", "phs_deg", "nt", "euclid_precond_level_hypre", "gmres_kdim",
                          "n_iter"):
                out[name] = int(v)
            else:
                out[name] = float(v)
        return out

    def verify_parameters(self):
        """parameters.cpp:82-120 (the mesh-file checks do not apply to in-memory clouds)."""
        if self.poly_deg < 2 or self.poly_deg > 15:
            raise capi.MemphysError(capi.MP_BAD_ARG, f"poly_deg should be in range [2, 15]; "
                                                     f"current value: {self.poly_deg}")
        if self.phs_deg not in (3, 5, 7, 9, 11):
            raise capi.MemphysError(capi.MP_BAD_ARG, f"phs_deg should be 3, 5, 7, 9, or 11; "
                                                     f"current value: {self.phs_deg}")
        self.solver_type = self.solver_type.lower()
        if self.solver_type not in SOLVER_TYPES:
            raise capi.MemphysError(capi.MP_BAD_ARG,
                                    f"solver_type should be one of {sorted(SOLVER_TYPES)}; "
                                    f"current value: {self.solver_type}")

    def calc_cloud_num_points(self):
        self.num_poly_terms = capi.lib().mp_num_poly_terms(self.dimension, self.poly_deg)
        self.cloud_size = capi.lib().mp_cloud_size(self.dimension, self.poly_deg,
                                                   self.cloud_size_multiplier)

    def calc_polynomial_term_exponents(self):
        e = np.zeros(self.num_poly_terms * self.dimension, np.int32)
        check(capi.lib().mp_poly_exponents(self.dimension, self.poly_deg, ptr(e)),
              "calc_polynomial_term_exponents")
        self.polynomial_term_exponents = e.reshape(self.num_poly_terms, self.dimension)

    def solver_cfg(self, **overrides) -> capi.SolverCfg:
        st = SOLVER_TYPES.get(self.solver_type, SOLVER_TYPES["cuda_bicgstab_amg"])
        kw = dict(tol=self.solver_tolerance, maxit=self.n_iter, **st)
        kw.update(overrides)
        return capi.solver_cfg(**kw)

    def integrator_cfg(self, **overrides) -> capi.SolverCfg:
        """The solver configuration of a time integrator's pressure solve.  The SOR
        sweeps of the `sor` type run through SOLVER only (the integrators capture their
        solves in CUDA graphs); an integrator given `sor` solves with BiCGSTAB + multigrid
        to the same tolerance and says so."""
        if self.solver_type == "sor" and "precond" not in overrides:
            print("PARAMETERS: solver_type sor -> the time integrator's pressure solve runs "
                  "BiCGSTAB + multigrid (SOR sweeps are available through SOLVER)")
            overrides = dict(overrides, precond=capi.MP_PRECOND_AMG)
        return self.solver_cfg(**overrides)


class POINTS:
    """class.hpp:96-140 for an in-memory cloud (the gmsh reader is not ported)."""

    def __init__(self, cloud: Cloud):
        self.cloud = cloud
        self.nv = cloud.nv
        self.dim = cloud.dim
        self.xyz = np.ascontiguousarray(cloud.xyz, np.float64)
        self.boundary_flag = np.ascontiguousarray(cloud.boundary, np.uint8)
        self.normal = np.ascontiguousarray(cloud.normal, np.float64)
        self.order = None  # new index of every input node once a CLOUD reorders them

    def permute(self, a: np.ndarray) -> np.ndarray:
        """A per-node array of the input order in this POINTS' current order."""
        a = np.asarray(a)
        if self.order is None:
            return a
        out = np.empty_like(a)
        out[self.order] = a
        return out

    def _reorder(self, order: np.ndarray):
        # re_order_points (cloud.cpp:337-439): coordinates, normals and flags move to
        # their new rows on the GPU
        order = np.ascontiguousarray(order, np.int32)
        L = capi.lib()
        for name in ("xyz", "normal", "boundary_flag"):
            a = np.ascontiguousarray(getattr(self, name))
            out = np.empty_like(a)
            row = a.nbytes // self.nv
            check(L.mp_permute_rows(ptr(a), ptr(out), self.nv, row, ptr(order), None),
                  "mp_permute_rows")
            setattr(self, name, out)
        self.order = order if self.order is None else order[self.order]


class CLOUD:
    """CLOUD::CLOUD (cloud.cpp:29-48) on the GPU: stencils, weights, operators."""

    def __init__(self, points: POINTS, parameters: PARAMETERS, compute_cond: bool = True,
                 nb_col: np.ndarray | None = None, reorder: str | None = None):
        """reorder: None keeps the input order; "rcm" renumbers the points and stencils
        by reverse Cuthill-McKee as the reference's constructor always does
        (cloud.cpp:37, mp_order_rcm); "morton" by the GPU Z-order (mp_order_morton).
        Reordering permutes `points` in place (points.order, points.permute)."""
        self.points = points
        h = C.c_void_p()
        if reorder is not None:
            if reorder not in ("rcm", "morton"):
                raise ValueError(f"reorder must be None, 'rcm' or 'morton', not {reorder!r}")
            L = capi.lib()
            if nb_col is None:
                n = L.mp_cloud_size(points.dim, parameters.poly_deg,
                                    C.c_double(parameters.cloud_size_multiplier))
                nb_col = np.zeros((points.nv, n), np.int32)
                check(L.mp_knn_stencils(ptr(points.xyz), ptr(points.boundary_flag), points.nv,
                                        points.dim, n, ptr(nb_col), None), "mp_knn_stencils")
            nb = np.ascontiguousarray(nb_col, np.int32)
            order = np.zeros(points.nv, np.int32)
            if reorder == "rcm":
                check(L.mp_order_rcm(ptr(nb), points.nv, nb.shape[1], ptr(order)), "mp_order_rcm")
            else:
                check(L.mp_order_morton(ptr(points.xyz), points.nv, points.dim, ptr(order), None),
                      "mp_order_morton")
            nb_col = np.zeros_like(nb)
            check(L.mp_permute_stencils(ptr(nb), points.nv, nb.shape[1], ptr(order), ptr(nb_col),
                                        None), "mp_permute_stencils")
            points._reorder(order)
        if nb_col is None:
            rc = capi.lib().mp_cloud_create(ptr(points.xyz), ptr(points.boundary_flag), points.nv,
                                            points.dim, parameters.phs_deg, parameters.poly_deg,
                                            parameters.cloud_size_multiplier, int(compute_cond),
                                            None, C.byref(h))
        else:
            nb = np.ascontiguousarray(nb_col, np.int32)
            rc = capi.lib().mp_cloud_create_stencils(ptr(points.xyz), ptr(points.boundary_flag),
                                                     points.nv, points.dim, ptr(nb), nb.shape[1],
                                                     parameters.phs_deg, parameters.poly_deg,
                                                     int(compute_cond), None, C.byref(h))
        check(rc, "CLOUD")
        self.handle = h
        nv, n, dim = C.c_int(), C.c_int(), C.c_int()
        check(capi.lib().mp_cloud_info(h, C.byref(nv), C.byref(n), C.byref(dim)))
        self.nv, self.n, self.dim = nv.value, n.value, dim.value
        self.compute_cond = compute_cond
        self._ops = {}

    def fetch(self):
        """Copy out nb_points_row/col, grad_*_coeff, laplacian_coeff, cond_num_RBF."""
        nv, n = self.nv, self.n
        nb = np.zeros((nv, n), np.int32)
        w = {k: np.zeros((nv, n)) for k in ("gx", "gy", "lap")}
        if self.dim == 3:
            w["gz"] = np.zeros((nv, n))
        cond = np.zeros(nv) if self.compute_cond else None
        check(capi.lib().mp_cloud_get(self.handle, ptr(nb), ptr(w["gx"]), ptr(w["gy"]),
                                      ptr(w.get("gz")), ptr(w["lap"]), ptr(cond), None),
              "mp_cloud_get")
        self.nb_points_col = nb
        self.nb_points_row = np.arange(nv + 1, dtype=np.int32) * n
        self.grad_x_coeff, self.grad_y_coeff = w["gx"], w["gy"]
        self.grad_z_coeff = w.get("gz")
        self.laplacian_coeff = w["lap"]
        if cond is not None:
            self.cond_num_RBF = cond
            self.cond_num_RBF_max = float(cond.max())
            self.cond_num_RBF_min = float(cond.min())
            self.cond_num_RBF_avg = float(cond.mean())
        return self

    def operator(self, which: int, rows: int = capi.MP_ROWS_ALL,
                 precision: int = capi.MP_FP64) -> "Operator":
        key = (which, rows, precision)
        if key not in self._ops:
            h = C.c_void_p()
            check(capi.lib().mp_op_from_cloud(self.handle, which, rows, precision, C.byref(h)),
                  "mp_op_from_cloud")
            self._ops[key] = Operator(h, self.nv, self.nv, precision)
        return self._ops[key]

    def __del__(self):
        try:
            self._ops.clear()
            if getattr(self, "handle", None):
                capi.lib().mp_cloud_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class Operator:
    """An ELL operator handle (mp_op); `op @ x` mirrors `matrix * VectorXd`."""

    def __init__(self, handle, nrows, ncols, precision):
        self.handle, self.nrows, self.ncols, self.precision = handle, nrows, ncols, precision

    @classmethod
    def from_ell(cls, cols: np.ndarray, vals: np.ndarray, ncols: int | None = None,
                 precision: int = capi.MP_FP64) -> "Operator":
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        nrows, width = cols.shape
        h = C.c_void_p()
        check(capi.lib().mp_op_create_ell(nrows, ncols or nrows, width, ptr(cols), ptr(vals),
                                          precision, C.byref(h)), "mp_op_create_ell")
        return cls(h, nrows, ncols or nrows, precision)

    def apply(self, x, y=None, alpha=1.0, beta=0.0, stream=None):
        dt = np.float64 if self.precision == capi.MP_FP64 else np.float32
        if y is None:
            y = np.zeros(self.nrows, dt)
        if isinstance(x, np.ndarray):
            x = np.ascontiguousarray(x, dt)
        check(capi.lib().mp_op_apply(self.handle, ptr(x), ptr(y), alpha, beta, stream),
              "mp_op_apply")
        return y

    def __matmul__(self, x):
        return self.apply(x)

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                capi.lib().mp_op_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class SOLVER:
    """SOLVER (solver.cpp): init() + general_solve() for the pressure operator."""

    def init(self, points: POINTS, cloud: CLOUD, parameters: PARAMETERS, dirichlet_flag,
             unsteady_term_coeff: float, conv_term_coeff: float, diff_term_coeff: float,
             log_flag: bool = True, **cfg_overrides):
        self.log_flag = log_flag
        self.cfg = parameters.solver_cfg(**cfg_overrides)
        self.dirichlet = np.ascontiguousarray(dirichlet_flag, np.uint8)
        h = C.c_void_p()
        check(capi.lib().mp_ppe_create(cloud.handle, ptr(points.boundary_flag), ptr(self.dirichlet),
                                       ptr(points.normal), unsteady_term_coeff, conv_term_coeff,
                                       diff_term_coeff, C.byref(self.cfg), C.byref(h)),
              "SOLVER::init")
        self.handle = h
        self.system_size = capi.lib().mp_ppe_system_size(h)
        self.nv = points.nv
        return self

    def general_solve(self, points, parameters, field_new, field_old, rhs):
        """solver.cpp:283-363: field_new = solve(rhs) from field_old; logs into parameters;
        the regularisation alpha is copied back into field_old (:361-362)."""
        x = np.array(field_old, np.float64, copy=True)
        b = np.ascontiguousarray(rhs, np.float64)
        it, rr, ar = C.c_int(), C.c_double(), C.c_double()
        rc = capi.lib().mp_ppe_solve(self.handle, ptr(b), ptr(x), C.byref(it), C.byref(rr),
                                     C.byref(ar), None)
        field_new[:] = x
        if self.cfg.precond == capi.MP_PRECOND_SOR:
            # solver.cpp:352-356: the SOR branch logs nothing into the parameters and
            # returns after its sweeps whether or not they reached the tolerance
            self.last_sor = (it.value, rr.value, rc)
            if rc not in (capi.MP_OK, capi.MP_NOT_CONVERGED):
                check(rc, "SOLVER::general_solve")
            return it.value, rr.value
        if self.log_flag:
            parameters.rel_res_log.append(rr.value)
            parameters.abs_res_log.append(ar.value)
            parameters.n_iter_actual.append(it.value)
            if self.system_size == points.nv + 1:
                parameters.regul_alpha_log.append(float(x[-1]))
        if self.system_size == points.nv + 1:
            field_old[self.system_size - 1] = x[-1]
        check(rc, "SOLVER::general_solve")
        return it.value, rr.value

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                capi.lib().mp_ppe_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class FRACTIONAL_STEP_1:
    """fractional_step_1.cpp: hat-velocity projection method on the GPU."""

    def __init__(self, points: POINTS, cloud: CLOUD, parameters: PARAMETERS, u_dirichlet_flag,
                 v_dirichlet_flag, p_dirichlet_flag, temporal_order: int,
                 w_dirichlet_flag=None, use_graph: bool = True, **cfg_overrides):
        self.dim = points.dim
        self.nv = points.nv
        self.use_graph = use_graph
        self.flags = [np.ascontiguousarray(f, np.uint8) for f in
                      (u_dirichlet_flag, v_dirichlet_flag,
                       w_dirichlet_flag if w_dirichlet_flag is not None else u_dirichlet_flag,
                       p_dirichlet_flag)]
        self.cfg = capi.Fs1Cfg(parameters.rho, parameters.mu, parameters.dt or 0.0,
                               temporal_order)
        self.scfg = parameters.integrator_cfg(**cfg_overrides)
        h = C.c_void_p()
        check(capi.lib().mp_fs1_create(cloud.handle, ptr(points.boundary_flag), ptr(points.normal),
                                       ptr(self.flags[0]), ptr(self.flags[1]),
                                       ptr(self.flags[2]) if self.dim == 3 else None,
                                       ptr(self.flags[3]), C.byref(self.cfg), C.byref(self.scfg),
                                       C.byref(h)), "FRACTIONAL_STEP_1")
        self.handle = h
        self.system_size = capi.lib().mp_fs1_system_size(h)
        self.cloud = cloud  # keep the cloud alive as long as the step object

    def _vec_ptrs(self, arrs):
        return (C.c_void_p * self.dim)(*[ptr(a).value for a in arrs])

    def set_state(self, vel, p, it=0):
        vel = [np.ascontiguousarray(v, np.float64) for v in vel]
        p = np.ascontiguousarray(p, np.float64)
        check(capi.lib().mp_fs1_set_state(self.handle, self._vec_ptrs(vel), ptr(p), it, None),
              "mp_fs1_set_state")

    def get_state(self):
        vel = [np.zeros(self.nv) for _ in range(self.dim)]
        p = np.zeros(self.system_size)
        check(capi.lib().mp_fs1_get_state(self.handle, self._vec_ptrs(vel), ptr(p), None),
              "mp_fs1_get_state")
        return vel, p

    def step(self, nsteps=1, stream=None):
        check(capi.lib().mp_fs1_step(self.handle, nsteps, int(self.use_graph), stream),
              "mp_fs1_step")

    def single_timestep_2d(self, points, cloud, parameters, u_new, v_new, p_new, u_old, v_old,
                           p_old, it):
        """fractional_step_1.cpp:52-63 with the reference's argument order."""
        if len(p_new) != self.system_size:
            raise capi.MemphysError(capi.MP_BAD_ARG, "p_new must have system_size entries")
        # keep every converted array referenced until the call returns
        uo = np.ascontiguousarray(u_old, np.float64)
        vo_ = np.ascontiguousarray(v_old, np.float64)
        po = np.ascontiguousarray(p_old, np.float64)
        vn = self._vec_ptrs([u_new, v_new])
        vo = self._vec_ptrs([uo, vo_])
        rc = capi.lib().mp_fs1_single_timestep(self.handle, vn, ptr(p_new), vo, ptr(po), it, None)
        iters, rr, ar, al = self.last_stats()
        parameters.rel_res_log.append(rr)
        parameters.abs_res_log.append(ar)
        parameters.n_iter_actual.append(iters)
        if self.system_size == self.nv + 1:
            parameters.regul_alpha_log.append(al)
            p_old[self.system_size - 1] = p_new[self.system_size - 1]
        check(rc, "FRACTIONAL_STEP_1::single_timestep_2d")

    def last_stats(self):
        it, rr, ar, al = C.c_int(), C.c_double(), C.c_double(), C.c_double()
        check(capi.lib().mp_fs1_last_stats(self.handle, C.byref(it), C.byref(rr), C.byref(ar),
                                           C.byref(al)), "mp_fs1_last_stats")
        return it.value, rr.value, ar.value, al.value

    def log(self, first, count):
        """Per-step logs: iterations, relres, abs res, alpha, initial relres, refinements."""
        out = np.zeros((count, 8))
        check(capi.lib().mp_fs1_log(self.handle, first, count, ptr(out)), "mp_fs1_log")
        return out

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                capi.lib().mp_fs1_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class SEMI_IMPLICIT_SPLIT_SOLVER:
    """SEMI_IMPLICIT_SPLIT_SOLVER (semi_implicit_split_solver.cpp:22-50, 2D) on the GPU
    (mp_sis_*).  The velocity matrices are solved by BiCGSTAB with a Jacobi
    preconditioner rebuilt at every outer iteration (to the parameters' tolerance);
    the pressure correction by the solver type's configuration."""

    def __init__(self, points: POINTS, cloud: CLOUD, parameters: PARAMETERS, u_dirichlet_flag,
                 v_dirichlet_flag, p_dirichlet_flag, n_outer_iter: int,
                 iterative_tolerance: float, precond_freq_it: int, use_graph: bool = True,
                 **p_cfg):
        if parameters.dt is None or parameters.rho < 0 or parameters.mu < 0:  # check_bc :65-70
            raise capi.MemphysError(capi.MP_BAD_ARG, "set parameters.rho, mu and dt first")
        cfg = capi.SisCfg(parameters.rho, parameters.mu, parameters.dt, int(n_outer_iter),
                          float(iterative_tolerance), int(precond_freq_it))
        vel = parameters.solver_cfg(precond=capi.MP_PRECOND_JACOBI, precision=capi.MP_FP64)
        pc = parameters.integrator_cfg(**p_cfg)
        flags = [np.ascontiguousarray(f, np.uint8) for f in
                 (u_dirichlet_flag, v_dirichlet_flag, p_dirichlet_flag)]
        h = C.c_void_p()
        check(capi.lib().mp_sis_create(cloud.handle, ptr(points.boundary_flag), ptr(points.normal),
                                       ptr(flags[0]), ptr(flags[1]), ptr(flags[2]), C.byref(cfg),
                                       C.byref(vel), C.byref(pc), C.byref(h)), "mp_sis_create")
        self.handle = h
        self.cloud = cloud
        ns = C.c_int()
        check(capi.lib().mp_sis_system_size(h, C.byref(ns)))
        self.system_size = ns.value
        self.nv = points.nv
        self._itol = float(iterative_tolerance)
        check(capi.lib().mp_sis_set_graph(h, int(use_graph)))

    @property
    def iterative_tolerance(self) -> float:
        """The L1-change tolerance of the outer iteration; the reference's driver resets
        this public member before every step (eccentric_couette_flow_batch_ml.cpp:71-73)."""
        return self._itol

    @iterative_tolerance.setter
    def iterative_tolerance(self, value: float):
        check(capi.lib().mp_sis_set_tolerance(self.handle, float(value)), "iterative_tolerance")
        self._itol = float(value)

    def single_timestep_2d(self, u_new, v_new, p_new, u_old, v_old, p_old, it,
                           n_outer_iter_log=None, iterative_l1_err_log=None,
                           iterative_max_err_log=None):
        """single_timestep_2d (:376-421): the new fields into u_new, v_new, p_new
        (arrays of nv, nv and system_size entries, written in place); the logs, when
        given, get the outer iterations and the last L1 / max changes appended."""
        ns = self.system_size
        uo, vo = (np.ascontiguousarray(a, np.float64) for a in (u_old, v_old))
        po = np.ascontiguousarray(p_old, np.float64)
        if po.shape[0] != ns:  # :380-383
            po = np.zeros(ns)
        for a, m in ((u_new, self.nv), (v_new, self.nv), (p_new, ns)):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.shape == (m,)
                    and a.flags.c_contiguous):
                raise capi.MemphysError(capi.MP_BAD_ARG, "u_new, v_new, p_new: float64 arrays of "
                                                    f"{self.nv}, {self.nv}, {ns} entries")
        vin = (C.c_void_p * 2)(uo.ctypes.data, vo.ctypes.data)
        vout = (C.c_void_p * 2)(u_new.ctypes.data, v_new.ctypes.data)
        n, l1, mx = C.c_int(), C.c_double(), C.c_double()
        check(capi.lib().mp_sis_single_timestep(self.handle, vin, ptr(po), vout, ptr(p_new),
                                                int(it), C.byref(n), C.byref(l1), C.byref(mx),
                                                None), "mp_sis_single_timestep")
        if n_outer_iter_log is not None:
            n_outer_iter_log.append(n.value)
        if iterative_l1_err_log is not None:
            iterative_l1_err_log.append(l1.value)
        if iterative_max_err_log is not None:
            iterative_max_err_log.append(mx.value)
        return n.value, l1.value, mx.value

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                capi.lib().mp_sis_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class IMPLICIT_SCALAR_TRANSPORT_SOLVER:
    """IMPLICIT_SCALAR_TRANSPORT_SOLVER (implicit_scalar_transport_solver.cpp:22-41, 2D)
    on the GPU (mp_ist_*); with solver_log_flag the relative and absolute residuals
    and iterations of every solve are appended to rel_res_log, abs_res_log and
    n_iter_actual, as the reference appends them to its parameters."""

    def __init__(self, points: POINTS, cloud: CLOUD, parameters: PARAMETERS, dirichlet_flag,
                 precond_freq_it: int, unsteady_coeff: float, conv_coeff: float,
                 diff_coeff: float, solver_log_flag: bool = False, use_graph: bool = True):
        cfg = parameters.solver_cfg(precond=capi.MP_PRECOND_JACOBI, precision=capi.MP_FP64)
        flag = np.ascontiguousarray(dirichlet_flag, np.uint8)
        h = C.c_void_p()
        check(capi.lib().mp_ist_create(cloud.handle, ptr(points.boundary_flag), ptr(points.normal),
                                       ptr(flag), int(precond_freq_it), float(unsteady_coeff),
                                       float(conv_coeff), float(diff_coeff), C.byref(cfg),
                                       C.byref(h)), "mp_ist_create")
        self.handle = h
        self.cloud = cloud
        self.nv = points.nv
        self.solver_log_flag = solver_log_flag
        self.rel_res_log, self.abs_res_log, self.n_iter_actual = [], [], []
        check(capi.lib().mp_ist_set_graph(h, int(use_graph)))

    def single_timestep_2d(self, phi_new, phi_old, u_new, v_new, it):
        """single_timestep_2d (:136-174): phi_new (float64, nv entries) written in place."""
        if not (isinstance(phi_new, np.ndarray) and phi_new.dtype == np.float64
                and phi_new.shape == (self.nv,) and phi_new.flags.c_contiguous):
            raise capi.MemphysError(capi.MP_BAD_ARG, f"phi_new: float64 array of {self.nv} entries")
        po, u, v = (np.ascontiguousarray(a, np.float64) for a in (phi_old, u_new, v_new))
        n, rr = C.c_int(), C.c_double()
        check(capi.lib().mp_ist_single_timestep(self.handle, ptr(po), ptr(u), ptr(v), ptr(phi_new),
                                                int(it), C.byref(n), C.byref(rr), None),
              "mp_ist_single_timestep")
        if self.solver_log_flag:
            self.rel_res_log.append(rr.value)
            self.n_iter_actual.append(n.value)
        return n.value, rr.value

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                capi.lib().mp_ist_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class FRACTIONAL_STEP_FOURIER:
    """FRACTIONAL_STEP_FOURIER (fractional_step_fourier.cpp:22-68) on the GPU (mp_fsf_*):
    a 2D cloud extruded periodically in z over 2 nw + 1 planes of `period`; fields are
    (nv, 2 nw + 1) arrays."""

    def __init__(self, points: POINTS, cloud: CLOUD, parameters: PARAMETERS, u_dirichlet_flag,
                 v_dirichlet_flag, w_dirichlet_flag, p_dirichlet_flag, period: float, nw: int,
                 temporal_order: int, use_graph: bool = True, **cfg):
        flags = [np.ascontiguousarray(f, np.uint8) for f in
                 (u_dirichlet_flag, v_dirichlet_flag, w_dirichlet_flag, p_dirichlet_flag)]
        sc = parameters.integrator_cfg(**cfg)
        h = C.c_void_p()
        check(capi.lib().mp_fsf_create(cloud.handle, ptr(points.boundary_flag), ptr(points.normal),
                                       *[ptr(f) for f in flags], float(period), int(nw),
                                       int(temporal_order), float(parameters.rho),
                                       float(parameters.mu), float(parameters.dt or 0.0),
                                       C.byref(sc), C.byref(h)), "mp_fsf_create")
        self.handle = h
        self.cloud = cloud
        self.nv, self.N = points.nv, 2 * int(nw) + 1
        check(capi.lib().mp_fsf_set_graph(h, int(use_graph)))
        # numpy's C-ordered (nv, N) arrays are node-major; the library transposes them
        # to and from its plane-contiguous layout (Eigen's column-major) on the device
        check(capi.lib().mp_fsf_set_layout(h, 1), "mp_fsf_set_layout")

    def single_timestep(self, u_new, v_new, w_new, p_new, u_old, v_old, w_old, p_old, it):
        """single_timestep (:250-266): (nv, 2 nw + 1) float64 arrays; the new fields are
        written in place."""
        shape = (self.nv, self.N)
        olds = [np.ascontiguousarray(np.asarray(a, np.float64).reshape(shape)) for a in
                (u_old, v_old, w_old, p_old)]
        news = (u_new, v_new, w_new, p_new)
        # results straight into C-contiguous float64 (nv, N) outputs, through a
        # temporary otherwise
        outs = [a if (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.shape == shape
                      and a.flags.c_contiguous and a.flags.writeable) else np.empty(shape)
                for a in news]
        vin = (C.c_void_p * 3)(*[a.ctypes.data for a in olds[:3]])
        vout = (C.c_void_p * 3)(*[a.ctypes.data for a in outs[:3]])
        check(capi.lib().mp_fsf_single_timestep(self.handle, vin, ptr(olds[3]), vout,
                                                ptr(outs[3]), int(it), None),
              "mp_fsf_single_timestep")
        for dst, src in zip(news, outs):
            if dst is not src:
                dst[...] = src.reshape(np.shape(dst))

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                capi.lib().mp_fsf_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class MLP:
    """The learned pressure-increment network (mp_mlp): 64 -> 128 -> 128 -> 128 -> 1."""

    def __init__(self, seed: int = 1):
        h = C.c_void_p()
        check(capi.lib().mp_mlp_create(seed, C.byref(h)), "mp_mlp_create")
        self.handle = h
        self.n_params = capi.lib().mp_mlp_num_params()

    def params(self) -> np.ndarray:
        th = np.zeros(self.n_params, np.float32)
        check(capi.lib().mp_mlp_get_params(self.handle, ptr(th)), "mp_mlp_get_params")
        return th

    def set_params(self, theta):
        th = np.ascontiguousarray(theta, np.float32)
        check(capi.lib().mp_mlp_set_params(self.handle, ptr(th)), "mp_mlp_set_params")

    def forward(self, X) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32)
        y = np.zeros(X.shape[0], np.float32)
        check(capi.lib().mp_mlp_forward(self.handle, ptr(X), X.shape[0], ptr(y)), "mp_mlp_forward")
        return y

    def gradient(self, X, t):
        X = np.ascontiguousarray(X, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(self.n_params, np.float32)
        loss = C.c_double()
        check(capi.lib().mp_mlp_gradient(self.handle, ptr(X), ptr(t), X.shape[0], C.byref(loss),
                                         ptr(g)), "mp_mlp_gradient")
        return loss.value, g

    def train(self, X, t, epochs=5, batch=1024, lr=1e-3, seed=0):
        X = np.ascontiguousarray(X, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        loss = C.c_double()
        check(capi.lib().mp_mlp_train(self.handle, ptr(X), ptr(t), X.shape[0], epochs, batch, lr,
                                      seed, C.byref(loss)), "mp_mlp_train")
        return loss.value

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                capi.lib().mp_mlp_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


def attach_mlp(fs: "FRACTIONAL_STEP_1", mlp: MLP, sample_nodes=8192, capacity_steps=500,
               collect=True):
    check(capi.lib().mp_fs1_attach_mlp(fs.handle, mlp.handle, sample_nodes, capacity_steps,
                                       int(collect)), "mp_fs1_attach_mlp")
    fs.mlp = mlp


def train_mlp(fs: "FRACTIONAL_STEP_1", epochs=5, batch=4096, lr=1e-3, seed=0) -> float:
    loss = C.c_double()
    check(capi.lib().mp_fs1_train_mlp(fs.handle, epochs, batch, lr, seed, C.byref(loss)),
          "mp_fs1_train_mlp")
    return loss.value


def samples(fs: "FRACTIONAL_STEP_1"):
    """The recorded training samples (features X, targets t, node of each row)."""
    n = C.c_int()
    L = capi.lib()
    check(L.mp_fs1_samples(fs.handle, None, None, None, 0, C.byref(n)), "mp_fs1_samples")
    X = np.zeros((n.value, 64), np.float32)
    t = np.zeros(n.value, np.float32)
    nodes = np.zeros(n.value, np.int32)
    check(L.mp_fs1_samples(fs.handle, capi.ptr(X), capi.ptr(t), capi.ptr(nodes), n.value,
                           C.byref(n)), "mp_fs1_samples")
    return X, t, nodes


def set_guess(fs: "FRACTIONAL_STEP_1", guess: int):
    check(capi.lib().mp_fs1_set_guess(fs.handle, guess), "mp_fs1_set_guess")


def cavity_setup(nx: int, solver_type="cuda_bicgstab_amg", dt=None, rho=1.0, mu=0.01,
                 temporal_order=2, tol=1e-8, maxit=1000, seed=None, use_graph=True, **cfg):
    """The lid-driven cavity of the benchmark configurations, ready to step."""
    from . import clouds
    cl = clouds.cavity_2d(nx) if seed is None else clouds.cavity_2d(nx, seed=seed)
    prm = PARAMETERS(solver_type=solver_type, solver_tolerance=tol, n_iter=maxit)
    prm.rho, prm.mu = rho, mu
    prm.dt = dt if dt is not None else stable_dt(cl.h, mu / rho)
    pts = POINTS(cl)
    cld = CLOUD(pts, prm, compute_cond=False)
    fs = FRACTIONAL_STEP_1(pts, cld, prm, cl.u_dirichlet, cl.v_dirichlet, cl.p_dirichlet,
                           temporal_order, use_graph=use_graph, **cfg)
    p0 = np.zeros(fs.system_size)
    fs.set_state([cl.vel_bc[0], cl.vel_bc[1]], p0, 0)
    return cl, prm, pts, cld, fs


def calc_largest_magnitude_eigenvalue(op: "Operator", ncv: int = 30, tol: float = 1e-10,
                                      max_restarts: int = 300, seed: int = 1) -> complex:
    """calc_largest_magnitude_eigenvalue (general_functions.cpp:4-24): the eigenvalue of
    largest magnitude of an operator, by restarted Arnoldi on the GPU (mp_op_largest_eig)
    to a Ritz residual of tol * |lambda|; raises MemphysError(NOT_CONVERGED) otherwise, as
    the reference throws when Spectra does not converge."""
    re, im, nr = C.c_double(), C.c_double(), C.c_int()
    check(capi.lib().mp_op_largest_eig(op.handle, ncv, tol, max_restarts, seed, C.byref(re),
                                       C.byref(im), C.byref(nr), None),
          "calc_largest_magnitude_eigenvalue")
    return complex(re.value, im.value)


def largest_eig_magnitude(op: "Operator", **kw) -> float:
    return abs(calc_largest_magnitude_eigenvalue(op, **kw))


def calc_dt(cloud: CLOUD, u0: float, v0: float, w0: float, alpha: float, courant: float,
            parameters: PARAMETERS | None = None) -> float:
    """PARAMETERS::calc_dt (parameters.cpp:269-296): dt = Courant * 2 /
    (u0|l_x| + v0|l_y| [+ w0|l_z|] + alpha|l_L|) from the largest-magnitude eigenvalues.
    With `parameters` the eigenvalues are stored there as the reference stores them
    (grad_x_eigval_real/imag, ..., laplace_eigval_real/imag) and dt is set."""
    names = [("grad_x", capi.MP_GRAD_X, u0), ("grad_y", capi.MP_GRAD_Y, v0)]
    if cloud.dim == 3:
        names.append(("grad_z", capi.MP_GRAD_Z, w0))
    names.append(("laplace", capi.MP_LAPLACIAN, alpha))
    ev = 0.0
    for name, which, coef in names:
        lam = calc_largest_magnitude_eigenvalue(cloud.operator(which))
        if parameters is not None:
            setattr(parameters, f"{name}_eigval_real", lam.real)
            setattr(parameters, f"{name}_eigval_imag", lam.imag)
        ev += coef * abs(lam)
    dt = courant * 2.0 / ev
    if parameters is not None:
        parameters.Courant = courant
        parameters.dt = dt
    return dt


def stable_dt(h: float, nu: float, lid: float = 1.0, safety: float = 0.5) -> float:
    """A step inside the explicit limits of the AB2 projection step on these clouds:
    safety * min(0.5 h / u, 0.02 h^2 / nu).  The diffusion bound is the AB2 limit
    1 / (nu |lambda_L|) with |lambda_L| ~ 46 / h^2, the spectral radius of the
    PHS-RBF-FD Laplacian on the jittered cavity (power iteration at h = 1e-3);
    calc_dt computes the same bound from the actual eigenvalues."""
    return safety * min(0.5 * h / lid, 0.02 * h * h / nu)
