"""Fourier-z fractional-step oracle in numpy -- TEST INFRASTRUCTURE ONLY.

Restates FRACTIONAL_STEP_FOURIER (fractional_step_fourier.cpp, without the
temperature and body-force overloads) on complex (nv x N) coefficient
matrices exactly as the reference lays them out, all N columns included, with
each mode's pressure system solved by a direct sparse LU.

  __init__            :22-68   (+ set_p_coeff_eigen :119-172)
  dft / idft          general_functions.cpp:1106-1137 (the reference's matrices)
  calc_vel_source     :375-398
  calc_vel_hat        :326-345
  calc_pressure       :400-442
  calc_vel_corr       :444-552
  single_timestep     :250-266
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as sla

from . import ppe_assemble


class FSF:
    def __init__(self, cloud, nb_col, w, rho, mu, dt, u_dir, v_dir, w_dir, p_dir, period, nw,
                 temporal_order=2):
        nv, n = nb_col.shape
        self.nv, self.n, self.nb = nv, n, np.asarray(nb_col)
        self.rho, self.mu, self.dt, self.order = rho, mu, dt, temporal_order
        self.nw, self.N = nw, 2 * nw + 1
        self.w = w
        self.bnd = np.asarray(cloud.boundary, bool)
        self.normal = np.asarray(cloud.normal)
        self.dirs = [np.asarray(f, bool) for f in (u_dir, v_dir, w_dir)]
        self.pdir = np.asarray(p_dir, bool)
        rows = np.repeat(np.arange(nv), n)
        mk = lambda v: sp.csr_matrix((np.ascontiguousarray(v).ravel(), (rows, self.nb.ravel())),
                                     shape=(nv, nv))
        self.Gx, self.Gy, self.L = mk(w["gx"]), mk(w["gy"]), mk(w["lap"])
        b = self.bnd
        self.Gx_int = mk(np.where(b[:, None], 0.0, w["gx"]))
        self.Gy_int = mk(np.where(b[:, None], 0.0, w["gy"]))
        N = self.N
        k = np.zeros(N)
        for iw in range(N):
            k[iw] = iw * 2 * np.pi / period if iw <= nw else -k[N - iw]
        self.k, self.k2 = k, k * k
        r = np.arange(N)
        self.D = np.exp(-1j * 2.0 * np.pi * np.outer(r, r) / (N * period))
        self.ID = np.exp(1j * 2.0 * np.pi * np.outer(r, r) / (N * period)) / N
        self.full_neumann = not np.any(b & self.pdir)
        self.P = []
        for iw in range(nw + 1):
            border = iw == 0 and self.full_neumann
            rp, ci, val, ns = ppe_assemble(self.nb, w, cloud.boundary, p_dir, cloud.normal,
                                           unsteady=-self.k2[iw], bordered=border)
            self.P.append(sla.splu(sp.csr_matrix((val, ci, rp), shape=(ns, ns)).tocsc()))
        z = np.zeros((nv, N), complex)
        self.u_ft, self.v_ft, self.w_ft, self.p_ft = z.copy(), z.copy(), z.copy(), z.copy()
        self.s_old = [z.copy() for _ in range(3)]

    def dft(self, phi):
        nw = self.nw
        out = np.zeros((phi.shape[0], self.N), complex)
        out[:, : nw + 1] = phi @ self.D[:, : nw + 1]
        out[:, nw + 1:] = np.conj(out[:, 1: nw + 1])[:, ::-1]
        return out

    def idft(self, ft):
        nw = self.nw
        phi = np.outer(ft[:, 0].real, self.ID[0].real) - np.outer(ft[:, 0].imag, self.ID[0].imag)
        phi = phi + 2.0 * (ft[:, 1: nw + 1].real @ self.ID[1: nw + 1].real
                           - ft[:, 1: nw + 1].imag @ self.ID[1: nw + 1].imag)
        return phi

    def vel_source(self, u, v, w, phi_ft, phi):
        xy = self.Gx @ (u * phi) + self.Gy @ (v * phi)
        c_xy = self.dft(xy)
        c_z = self.dft(w * phi) * (1j * self.k)[None, :]
        src = -self.rho * (c_xy + c_z)
        return src + self.mu * ((self.L @ phi_ft) - phi_ft * self.k2[None, :])

    def single_timestep(self, u_old, v_old, w_old, p_old, it):
        rho, dt, nv, nw, N = self.rho, self.dt, self.nv, self.nw, self.N
        if it == 0:
            self.u_ft, self.v_ft = self.dft(u_old), self.dft(v_old)
            self.w_ft, self.p_ft = self.dft(w_old), self.dft(p_old)
        s = [self.vel_source(u_old, v_old, w_old, f, q) for f, q in
             ((self.u_ft, u_old), (self.v_ft, v_old), (self.w_ft, w_old))]
        olds = (self.u_ft, self.v_ft, self.w_ft)
        if self.order == 1 or it == 0:
            h = [o + (dt / rho) * si for o, si in zip(olds, s)]
        else:
            h = [o + (0.5 * dt / rho) * (3.0 * si - so) for o, si, so in zip(olds, s, self.s_old)]
        uh, vh, wh = h
        # calc_pressure
        ps = np.zeros((nv + 1, N), complex)
        ps[:nv] = self.Gx_int @ uh + self.Gy_int @ vh
        ps[:nv] = ps[:nv] + wh * (1j * self.k)[None, :]
        ps = ps * rho / dt
        b, nrm = self.bnd, self.normal
        for i in np.nonzero(b)[0]:
            if self.pdir[i]:
                ps[i] = self.p_ft[i]
            else:
                ps[i] = -rho * ((self.u_ft[i] - uh[i]) * nrm[i, 0]
                                + (self.v_ft[i] - vh[i]) * nrm[i, 1]) / dt
        p_new = np.zeros((nv, N), complex)
        for iw in range(nw + 1):
            if iw == 0 and self.full_neumann:
                x = self.P[0].solve(ps[:, 0].real.copy())
                p_new[:, 0] = x[:nv]
            else:
                p_new[:, iw] = (self.P[iw].solve(ps[:nv, iw].real.copy())
                                + 1j * self.P[iw].solve(ps[:nv, iw].imag.copy()))
            if iw > 0:
                p_new[:, N - iw] = np.conj(p_new[:, iw])
        # calc_vel_corr
        c = dt / rho
        un = uh - (self.Gx @ p_new) * c
        vn = vh - (self.Gy @ p_new) * c
        wn = wh - (p_new * (1j * self.k)[None, :]) * c
        w_, nb = self.w, self.nb
        for q, (new, old) in enumerate(((un, self.u_ft), (vn, self.v_ft), (wn, self.w_ft))):
            for i in np.nonzero(b & ~self.pdir)[0]:
                if self.dirs[q][i]:
                    new[i] = old[i]
                    continue
                cf = w_["gx"][i] * nrm[i, 0] + w_["gy"][i] * nrm[i, 1]
                for iw in range(N):
                    rhs = 0.0 + 0.0j
                    diag = 0.0
                    for kk in range(self.n):
                        j = nb[i, kk]
                        if j == i:
                            diag = cf[kk]
                        else:
                            rhs = rhs - cf[kk] * new[j, iw]
                    new[i, iw] = rhs / diag
        self.u_ft, self.v_ft, self.w_ft, self.p_ft = un, vn, wn, p_new
        self.s_old = s
        return self.idft(un), self.idft(vn), self.idft(wn), self.idft(p_new)
