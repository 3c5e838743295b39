"""Fractional-step oracle in numpy -- TEST INFRASTRUCTURE ONLY.

Restates FRACTIONAL_STEP_1 (fractional_step_1.cpp) with the pressure solved
by a direct sparse LU, which is the reference's `eigen_direct` solver branch
(solver.cpp:55-60, 323-336: Eigen::SparseLU with COLAMD ordering).  SuperLU
(scipy) with partial pivoting plays the role of Eigen::SparseLU: the solution
of the same bordered system to rounding, independent of any iterative
tolerance, so it is the reference the GPU BiCGSTAB is checked against.

  FS1.__init__        fractional_step_1.cpp:22-50  (+ SOLVER::init, solver.cpp:14-79)
  FS1.calc_vel_hat    fractional_step_1.cpp:120-134
  FS1.calc_pressure   fractional_step_1.cpp:136-151
  FS1.calc_vel_corr   fractional_step_1.cpp:153-209
  FS1.extras          fractional_step_1.cpp:211-222
The reference steps 2D only; dim == 3 adds the w component with the same steps.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as sla

from . import ppe_assemble


class FS1:
    def __init__(self, cloud, nb_col, w, rho, mu, dt, temporal_order=2, factor=True):
        """factor=False skips the direct factorisation: the instance then only forms
        the right-hand sides and corrections around pressures supplied by the caller
        (step_with_pressure), which is how the full-size configurations are checked."""
        nv, n = nb_col.shape
        self.nv, self.dim = nv, cloud.dim
        self.rho, self.mu, self.dt, self.order = rho, mu, dt, temporal_order
        rows = np.repeat(np.arange(nv), n)
        mk = lambda v: sp.csr_matrix((np.ascontiguousarray(v).ravel(), (rows, nb_col.ravel())),
                                     shape=(nv, nv))
        names = ["gx", "gy", "gz"][: self.dim]
        self.G = [mk(w[k]) for k in names]
        self.L = mk(w["lap"])
        b = np.asarray(cloud.boundary, bool)
        self.G_int = [mk(np.where(b[:, None], 0.0, w[k])) for k in names]
        self.bnd = b
        self.normal = np.asarray(cloud.normal)
        self.vdir = [np.asarray(cloud.u_dirichlet, bool), np.asarray(cloud.v_dirichlet, bool)]
        if self.dim == 3:
            self.vdir.append(np.asarray(cloud.w_dirichlet, bool))
        self.pdir = np.asarray(cloud.p_dirichlet, bool)
        self.nb, self.w = nb_col, w
        rp, ci, val, ns = ppe_assemble(nb_col, w, cloud.boundary, cloud.p_dirichlet, cloud.normal)
        self.A = sp.csr_matrix((val, ci, rp), shape=(ns, ns))
        self.nsys = ns
        self.lu = sla.splu(self.A.tocsc()) if factor else None
        self.src_old = [np.zeros(nv) for _ in range(self.dim)]
        self.src_oldold = [np.zeros(nv) for _ in range(self.dim)]

    def calc_vel_hat(self, vel, it):
        hat = []
        for d in range(self.dim):
            q = vel[d]
            conv = -(vel[0] * (self.G[0] @ q))
            for e in range(1, self.dim):
                conv = conv - vel[e] * (self.G[e] @ q)
            src = self.rho * conv + self.mu * (self.L @ q)
            self.src_old[d] = src
            if self.order == 1 or it == 0:
                hat.append(q + (self.dt / self.rho) * src)
            else:
                hat.append(q + (self.dt / self.rho) * (1.5 * src - 0.5 * self.src_oldold[d]))
        return hat

    def pressure_rhs(self, vel, hat, p_old):
        """fractional_step_1.cpp:136-149: the right-hand side of the pressure system."""
        nv = self.nv
        s = self.G_int[0] @ hat[0]
        for d in range(1, self.dim):
            s = s + self.G_int[d] @ hat[d]
        src = np.zeros(self.nsys)
        src[:nv] = s * self.rho / self.dt
        b = self.bnd
        pd = b & self.pdir
        src[:nv][pd] = p_old[:nv][pd]
        nm = b & ~self.pdir
        acc = (vel[0] - hat[0]) * self.normal[:, 0]
        for d in range(1, self.dim):
            acc = acc + (vel[d] - hat[d]) * self.normal[:, d]
        src[:nv][nm] = (-self.rho * acc / self.dt)[nm]
        if self.nsys == nv + 1:
            src[nv] = 0.0
        return src

    def calc_pressure(self, vel, hat, p_old):
        src = self.pressure_rhs(vel, hat, p_old)
        p = self.lu.solve(src)
        self.last_rhs = src
        self.last_relres = np.linalg.norm(self.A @ p - src) / np.linalg.norm(src)
        return p

    def calc_vel_corr(self, vel, hat, p):
        nv = self.nv
        new = []
        for d in range(self.dim):
            q = hat[d] - (self.dt * (self.G[d] @ p[:nv])) / self.rho
            fix = self.bnd & ~self.pdir
            q[fix & self.vdir[d]] = vel[d][fix & self.vdir[d]]
            for i in np.nonzero(fix & ~self.vdir[d])[0]:
                cols = self.nb[i]
                cf = sum(self.w[k][i] * self.normal[i, e]
                         for e, k in enumerate(["gx", "gy", "gz"][: self.dim]))
                self_ = cols == i
                q[i] = -(cf[~self_] * q[cols[~self_]]).sum() / cf[self_][0]
            new.append(q)
        return new

    def step_with_pressure(self, vel, p, it, p_new):
        """One step whose pressure solve is replaced by `p_new` (a solution from
        elsewhere): returns ||A p_new - b|| / ||b|| with the oracle's own A and b
        (recomputed in FP64), then advances (vel, p) in place with that pressure."""
        hat = self.calc_vel_hat(vel, it)
        b = self.pressure_rhs(vel, hat, p)
        relres = np.linalg.norm(self.A @ p_new - b) / np.linalg.norm(b)
        new = self.calc_vel_corr(vel, hat, p_new)
        if self.order == 2:
            self.src_oldold = [s.copy() for s in self.src_old]
        for d in range(self.dim):
            vel[d][:] = new[d]
        p[:] = p_new
        return relres

    def step(self, vel, p, it):
        """Advance (vel, p) by one step in place; returns the pressure relative residual."""
        hat = self.calc_vel_hat(vel, it)
        pn = self.calc_pressure(vel, hat, p)
        new = self.calc_vel_corr(vel, hat, pn)
        if self.order == 2:
            self.src_oldold = [s.copy() for s in self.src_old]
        for d in range(self.dim):
            vel[d][:] = new[d]
        p[:] = pn
        return self.last_relres
