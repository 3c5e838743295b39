"""Semi-implicit split solver oracle in numpy -- TEST INFRASTRUCTURE ONLY.

Restates SEMI_IMPLICIT_SPLIT_SOLVER (semi_implicit_split_solver.cpp, 2D) with
every linear system solved by a direct sparse LU (SuperLU), so that the oracle
is the solution of the reference's equations to rounding, independent of the
iterative tolerances (the reference solves the velocity systems with Eigen's
BiCGSTAB + ILUT and the pressure correction with its configured solver).

  SIS.__init__            :22-50   (+ SOLVER::init for the pressure, solver.cpp:14-79)
  SIS.vel_matrix          :218-243, 245-324 (interior rows from the current u, v)
  SIS.calc_vel            :73-129  (no body force)
  SIS.calc_pressure       :131-186 (boundary rows in index order, as the loop runs)
  SIS.calc_vel_corr       :188-204
  SIS.single_timestep_2d  :376-421 (+ extras :206-216)
  IST                     implicit_scalar_transport_solver.cpp:22-174 (one direct solve per step)
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as sla

from . import ppe_assemble

A1, A2, A3 = 1.5, -2.0, 0.5  # BDF2 (class.hpp:414)


class SIS:
    def __init__(self, cloud, nb_col, w, rho, mu, dt, u_dir, v_dir, p_dir, n_outer_iter,
                 iterative_tolerance):
        nv, n = nb_col.shape
        self.nv, self.n, self.nb = nv, n, np.asarray(nb_col)
        self.rho, self.mu, self.dt = rho, mu, dt
        self.n_outer, self.itol = n_outer_iter, iterative_tolerance
        self.w = w
        self.bnd = np.asarray(cloud.boundary, bool)
        self.normal = np.asarray(cloud.normal)
        self.udir, self.vdir = np.asarray(u_dir, bool), np.asarray(v_dir, bool)
        self.pdir = np.asarray(p_dir, bool)
        rows = np.repeat(np.arange(nv), n)
        self.rows = rows
        mk = lambda v: sp.csr_matrix((np.ascontiguousarray(v).ravel(), (rows, self.nb.ravel())),
                                     shape=(nv, nv))
        b = self.bnd
        self.Gx, self.Gy, self.L = mk(w["gx"]), mk(w["gy"]), mk(w["lap"])
        self.Gx_int = mk(np.where(b[:, None], 0.0, w["gx"]))
        self.Gy_int = mk(np.where(b[:, None], 0.0, w["gy"]))
        rp, ci, val, ns = ppe_assemble(self.nb, w, cloud.boundary, p_dir, cloud.normal)
        self.nsys = ns
        self.P = sla.splu(sp.csr_matrix((val, ci, rp), shape=(ns, ns)).tocsc())
        self.uoo = np.zeros(nv)
        self.voo = np.zeros(nv)

    def vel_matrix(self, u, v, dirflag, unsteady):
        """Interior rows -mu L + rho(u_i Gx + v_i Gy) + unsteady rho/dt on the diagonal;
        boundary rows identity (Dirichlet) or n . G."""
        nb, w, b = self.nb, self.w, self.bnd
        vals = -self.mu * w["lap"] + (u[:, None] * self.rho) * w["gx"] + (v[:, None] * self.rho) * w["gy"]
        vals = vals + np.where(nb == np.arange(self.nv)[:, None], unsteady * self.rho / self.dt, 0.0)
        nrm = self.normal
        neu = nrm[:, :1] * w["gx"] + nrm[:, 1:2] * w["gy"]
        dirrow = np.where(nb == np.arange(self.nv)[:, None], 1.0, 0.0)
        vals = np.where(b[:, None], np.where(dirflag[:, None], dirrow, neu), vals)
        return sp.csr_matrix((vals.ravel(), (self.rows, nb.ravel())), shape=(self.nv, self.nv))

    def single_timestep_2d(self, u_old, v_old, p_old, it):
        nv, rho, dt, mu = self.nv, self.rho, self.dt, self.mu
        bdf1 = it == 0
        a1 = 1.0 if bdf1 else A1
        u, v, p = u_old.copy(), v_old.copy(), p_old.copy()
        l1 = mx = 0.0
        outer = 0
        for outer in range(1, self.n_outer + 1):
            ui, vi = u.copy(), v.copy()
            Mu = self.vel_matrix(u, v, self.udir, a1)
            Mv = self.vel_matrix(u, v, self.vdir, a1)
            # calc_vel
            gxp, gyp = self.Gx_int @ p[:nv], self.Gy_int @ p[:nv]
            if bdf1:
                su = (rho / dt) * u_old - gxp
                sv = (rho / dt) * v_old - gyp
            else:
                su = -((A2 * rho / dt) * u_old) - ((A3 * rho / dt) * self.uoo) - gxp
                sv = -((A2 * rho / dt) * v_old) - ((A3 * rho / dt) * self.voo) - gyp
            b = self.bnd
            su = np.where(b, np.where(self.udir, u_old, 0.0), su)
            sv = np.where(b, np.where(self.vdir, v_old, 0.0), sv)
            u = sla.spsolve(Mu.tocsc(), su)
            v = sla.spsolve(Mv.tocsc(), sv)
            # calc_pressure
            ps = np.zeros(self.nsys)
            ps[:nv] = (self.Gx_int @ u + self.Gy_int @ v) * (a1 * rho / dt)
            pp = self.P.solve(ps)
            p = p + pp
            if bdf1:
                tu, tv = u - u_old, v - v_old
            else:
                tu = A1 * u + A2 * u_old + A3 * self.uoo
                tv = A1 * v + A2 * v_old + A3 * self.voo
            mom_x = -rho * (u * (self.Gx @ u) + v * (self.Gy @ u)) + mu * (self.L @ u) - (rho / dt) * tu
            mom_y = -rho * (u * (self.Gx @ v) + v * (self.Gy @ v)) + mu * (self.L @ v) - (rho / dt) * tv
            nrm, w, nb = self.normal, self.w, self.nb
            for i in np.nonzero(b & ~self.pdir)[0]:
                rhs = mom_x[i] * nrm[i, 0] + mom_y[i] * nrm[i, 1]
                diag = 0.0
                for k in range(self.n):
                    j = nb[i, k]
                    cf = w["gx"][i, k] * nrm[i, 0] + w["gy"][i, k] * nrm[i, 1]
                    if j == i:
                        diag = cf
                    else:
                        rhs -= cf * p[j]
                p[i] = rhs / diag
            # calc_vel_corr
            f = dt / (a1 * rho)
            u = u - (self.Gx_int @ pp[:nv]) * f
            v = v - (self.Gy_int @ pp[:nv]) * f
            l1 = np.abs(u - ui).sum() / (2 * nv) + np.abs(v - vi).sum() / (2 * nv)
            mx = np.abs(u - ui).max() / 2 + np.abs(v - vi).max() / 2
            if l1 <= self.itol:
                break
        self.uoo, self.voo = u_old.copy(), v_old.copy()
        return u, v, p, outer, l1, mx


class IST:
    """IMPLICIT_SCALAR_TRANSPORT_SOLVER: interior rows diff L + conv (u_i Gx + v_i Gy)
    + a1 unsteady on the diagonal, boundary rows identity / n . G, BDF1 then BDF2."""

    def __init__(self, cloud, nb_col, w, dirichlet, unsteady, conv, diff):
        self.nb, self.w = np.asarray(nb_col), w
        self.nv, self.n = self.nb.shape
        self.bnd = np.asarray(cloud.boundary, bool)
        self.normal = np.asarray(cloud.normal)
        self.dir = np.asarray(dirichlet, bool)
        self.unsteady, self.conv, self.diff = unsteady, conv, diff
        self.rows = np.repeat(np.arange(self.nv), self.n)
        self.poo = np.zeros(self.nv)

    def single_timestep_2d(self, phi_old, u, v, it):
        nb, w, b = self.nb, self.w, self.bnd
        a1 = 1.0 if it == 0 else A1
        vals = self.diff * w["lap"] + (u[:, None] * self.conv) * w["gx"] + (v[:, None] * self.conv) * w["gy"]
        eye = nb == np.arange(self.nv)[:, None]
        vals = vals + np.where(eye, a1 * self.unsteady, 0.0)
        neu = self.normal[:, :1] * w["gx"] + self.normal[:, 1:2] * w["gy"]
        vals = np.where(b[:, None], np.where(self.dir[:, None], eye * 1.0, neu), vals)
        M = sp.csr_matrix((vals.ravel(), (self.rows, nb.ravel())), shape=(self.nv, self.nv))
        if it == 0:
            src = self.unsteady * phi_old
        else:
            src = -((A2 * self.unsteady) * phi_old) - ((A3 * self.unsteady) * self.poo)
        src = np.where(b, np.where(self.dir, phi_old, 0.0), src)
        phi = sla.spsolve(M.tocsc(), src)
        self.poo = phi_old.copy()
        return phi
