"""GPU: concentric Couette flow on the reference's annulus meshes against the
analytic profile.

The reference's driver checks its concentric runs against CONC_ANALYTICAL
(examples/navier_stokes_2D/eccentric_couette_flow_batch_ml_func.cpp:285-303):
u_theta(r) = C1 r + C2 / r, eta = r_i / r_o, C1 = -(omega_i eta^2 - omega_o) /
(1 - eta^2), C2 = r_i^2 (omega_i - omega_o) / (1 - eta^2).  Here every stage runs
on the GPU: the kNN stencils and PHS weights of the meshes' nodes (fixtures from
tests/golden/make_golden.py: ecc_ratio_0.0_r_i_0.5, n = 100 and 150), then
SEMI_IMPLICIT_SPLIT_SOLVER (the solver that driver uses) to steady state with the
inner wall turning at omega_i = 1, the outer at rest and pressure Neumann on
both walls (a bordered pressure system).  The velocity must approach the
analytic profile as closely as the oracle's does (tests/test_couette.py:
3.95e-3 and 1.25e-3 of omega r_i) and converge faster than linearly.
"""
import os

import numpy as np
import pytest

from memphys_b200 import clouds, meshless

pytestmark = pytest.mark.gpu

RI, RO, OMEGA = 0.5, 1.0, 1.0


def gpu_couette_error(golden_dir, n):
    d = np.load(os.path.join(golden_dir, "couette_clouds.npz"))
    xyz, bnd, nrm = d[f"xyz_{n}"], d[f"boundary_{n}"], d[f"normal_{n}"]
    nv = len(xyz)
    r = np.sqrt((xyz ** 2).sum(1))
    inner = bnd & (r < 0.5 * (RI + RO))
    cl = clouds.Cloud(name=f"couette_{n}", xyz=xyz, boundary=bnd, normal=nrm, u_dirichlet=bnd,
                      v_dirichlet=bnd, p_dirichlet=np.zeros(nv, bool))
    # 1e-9: the velocity systems (I - dt mu L, dt mu / h^2 ~ 1e4) floor near 1e-10 in FP64
    prm = meshless.PARAMETERS(solver_type="cuda_bicgstab_amg", solver_tolerance=1e-9,
                              n_iter=5000)
    prm.rho, prm.mu, prm.dt = 1.0, 1.0, 0.2
    pts = meshless.POINTS(cl)
    cld = meshless.CLOUD(pts, prm, compute_cond=False)
    assert cld.n == 20
    sis = meshless.SEMI_IMPLICIT_SPLIT_SOLVER(pts, cld, prm, bnd, bnd, np.zeros(nv, bool), 20,
                                              1e-8, 1)
    assert sis.system_size == nv + 1
    u = np.where(inner, -OMEGA * xyz[:, 1], 0.0)
    v = np.where(inner, OMEGA * xyz[:, 0], 0.0)
    p = np.zeros(sis.system_size)
    outer = []
    for it in range(30):                              # t = 6, many viscous times
        un, vn, pn = np.zeros(nv), np.zeros(nv), np.zeros(sis.system_size)
        outer.append(sis.single_timestep_2d(un, vn, pn, u, v, p, it)[0])
        u, v, p = un, vn, pn
    eta = RI / RO
    c1 = -(OMEGA * eta * eta - 0.0) / (1 - eta * eta)
    c2 = RI * RI * (OMEGA - 0.0) / (1 - eta * eta)
    ut = c1 * r + c2 / r
    ua, va = -ut * xyz[:, 1] / r, ut * xyz[:, 0] / r
    assert np.array_equal(u[bnd], np.where(inner, -OMEGA * xyz[:, 1], 0.0)[bnd])
    return float(max(np.abs(u - ua).max(), np.abs(v - va).max()) / (RI * OMEGA)), outer


def test_gpu_concentric_couette_converges_to_analytic(mp_lib, golden_dir):
    e100, o100 = gpu_couette_error(golden_dir, 100)
    e150, o150 = gpu_couette_error(golden_dir, 150)
    print("max velocity error / (omega r_i): n_100 %.2e, n_150 %.2e" % (e100, e150))
    print("outer iterations per step:", o100, o150)
    assert e100 < 6e-3 and e150 < 2e-3
    assert e150 < 0.5 * e100
    # the oracle's errors on the same meshes (tests/test_couette.py): the GPU's stencils,
    # weights and solves leave the same discretisation error
    assert abs(e100 - 3.95e-3) <= 0.02 * 3.95e-3 and abs(e150 - 1.25e-3) <= 0.02 * 1.25e-3
