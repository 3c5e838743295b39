"""Concentric Couette flow against the analytic profile (CPU oracle).

The reference's driver checks its concentric runs against CONC_ANALYTICAL
(examples/navier_stokes_2D/eccentric_couette_flow_batch_ml_func.cpp:285-303):
u_theta(r) = C1 r + C2 / r with eta = r_i / r_o, C1 = -(omega_i eta^2 - omega_o)
/ (1 - eta^2), C2 = r_i^2 (omega_i - omega_o) / (1 - eta^2).  The semi-implicit
split solver oracle (the solver that driver uses) runs to steady state on the
reference's concentric meshes (r_i = 0.5, r_o = 1, inner wall turning at
omega_i = 1, outer at rest; fixtures from tests/golden/make_golden.py): the
velocity must approach the analytic profile, and faster than linearly as the
mesh is refined (the GPU solver matches this oracle to the solve tolerance,
tests/test_gpu_sis.py).
"""
import os
import types

import numpy as np

import oracle
from oracle import sis as osis

RI, RO, OMEGA = 0.5, 1.0, 1.0


def couette_error(golden_dir, n):
    d = np.load(os.path.join(golden_dir, "couette_clouds.npz"))
    xyz, bnd, nrm = d[f"xyz_{n}"], d[f"boundary_{n}"], d[f"normal_{n}"]
    nv = len(xyz)
    r = np.sqrt((xyz ** 2).sum(1))
    inner = bnd & (r < 0.5 * (RI + RO))
    cl = types.SimpleNamespace(boundary=bnd.astype(np.uint8), normal=nrm, nv=nv)
    nb = oracle.knn_stencils(xyz, bnd.astype(np.uint8), 20)
    w = oracle.cloud_weights(xyz, nb, 3, 3, cond=False)
    eta = RI / RO
    c1 = -(OMEGA * eta * eta - 0.0) / (1 - eta * eta)
    c2 = RI * RI * (OMEGA - 0.0) / (1 - eta * eta)
    ut = c1 * r + c2 / r
    ua, va = -ut * xyz[:, 1] / r, ut * xyz[:, 0] / r
    u = np.where(inner, -OMEGA * xyz[:, 1], 0.0)    # walls: Dirichlet, pressure all Neumann
    v = np.where(inner, OMEGA * xyz[:, 0], 0.0)
    sis = osis.SIS(cl, nb, w, 1.0, 1.0, 0.2, bnd, bnd, np.zeros(nv, bool), 20, 1e-10)
    p = np.zeros(sis.nsys)
    for it in range(30):                             # t = 6, many viscous times
        u, v, p, *_ = sis.single_timestep_2d(u, v, p, it)
    return float(max(np.abs(u - ua).max(), np.abs(v - va).max()) / (RI * OMEGA))


def test_concentric_couette_converges_to_analytic(golden_dir):
    e100, e150 = couette_error(golden_dir, 100), couette_error(golden_dir, 150)
    print("max velocity error / (omega r_i): n_100 %.2e, n_150 %.2e" % (e100, e150))
    assert e100 < 6e-3 and e150 < 2e-3
    assert e150 < 0.5 * e100    # measured 3.95e-3 -> 1.25e-3 for spacing / 1.47: third order
