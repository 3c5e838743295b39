"""The reference's `sor` solver type (SOLVER::SOR, solver.cpp:243-281) on the GPU.

  sweeps      after k multicolour sweeps (omega 1.4, unbordered system) the GPU
              iterate equals the oracle's multicolour SOR with the same greedy
              colouring, to 1e-10 relative (rounding of the row sums only)
  converged   on an implicit velocity-type system the GPU sweeps reach the
              tolerance and the direct solution to 1e-9
  integrators a time integrator given `sor` says so and solves by BiCGSTAB +
              multigrid; the C entry point refuses the SOR configuration there
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as sla

import oracle
from memphys_b200 import capi, clouds, meshless
from memphys_b200.capi import ptr

pytestmark = pytest.mark.gpu


def setup(cl, dirichlet, unsteady, diff, n_iter, tol):
    prm = meshless.PARAMETERS(solver_type="sor", solver_tolerance=tol, n_iter=n_iter)
    pts = meshless.POINTS(cl)
    cld = meshless.CLOUD(pts, prm, compute_cond=False).fetch()
    s = meshless.SOLVER().init(pts, cld, prm, dirichlet, unsteady, 0.0, diff, True)
    w = {"gx": cld.grad_x_coeff, "gy": cld.grad_y_coeff, "lap": cld.laplacian_coeff}
    rp, ci, val, ns = oracle.ppe_assemble(cld.nb_points_col, w, cl.boundary, dirichlet,
                                          cl.normal, unsteady=unsteady, diff=diff,
                                          bordered=False)
    assert s.system_size == ns == cl.nv  # solver.cpp:30-31: no border for SOR
    return prm, pts, s, (rp, ci, val)


@pytest.mark.parametrize("make", [lambda: clouds.cavity_2d(24, seed=3),
                                  lambda: clouds.channel_2d(0.05, seed=1)])
def test_sor_sweeps_match_oracle(mp_lib, make):
    cl = make()
    prm, pts, s, (rp, ci, val) = setup(cl, cl.p_dirichlet, 0.0, 1.0, 30, 1e-300)
    rng = np.random.default_rng(7)
    b = rng.standard_normal(cl.nv)
    x0 = rng.standard_normal(cl.nv)
    x_old, x = x0.copy(), np.zeros(cl.nv)
    it, rr = s.general_solve(pts, prm, x, x_old, b)
    assert it == 30 and s.last_sor[2] == capi.MP_NOT_CONVERGED
    assert prm.rel_res_log == []  # the SOR branch logs nothing (solver.cpp:352-356)
    colour = oracle.sor_colouring(rp, ci, val, cl.nv)
    ref = oracle.sor_sweeps(rp, ci, val, b, x0, 1.4, 30, colour)
    print(f"{cl.name}: {colour.max() + 1} colours, relres after 30 sweeps {rr:.3e}")
    assert np.abs(x - ref).max() <= 1e-10 * np.abs(ref).max()
    A = sp.csr_matrix((val, ci, rp), shape=(cl.nv, cl.nv))
    assert rr == pytest.approx(np.linalg.norm(A @ x - b) / np.linalg.norm(b), rel=1e-9)


def test_sor_converges_to_direct_solution(mp_lib):
    cl = clouds.cavity_2d(32, seed=4)
    prm, pts, s, (rp, ci, val) = setup(cl, cl.u_dirichlet, 2000.0, -1.0, 5000, 1e-12)
    A = sp.csr_matrix((val, ci, rp), shape=(cl.nv, cl.nv))
    b = np.random.default_rng(8).standard_normal(cl.nv)
    x_old, x = np.zeros(cl.nv), np.zeros(cl.nv)
    it, rr = s.general_solve(pts, prm, x, x_old, b)
    assert s.last_sor[2] == capi.MP_OK and rr <= 1e-12 and it < 5000 and it % 10 == 0
    assert np.linalg.norm(A @ x - b) <= 1.01e-12 * np.linalg.norm(b)
    xd = sla.spsolve(A.tocsc(), b)
    assert np.abs(x - xd).max() <= 1e-9 * np.abs(xd).max()


def test_sor_in_time_integrators(mp_lib, capsys):
    cl = clouds.cavity_2d(16, seed=2)
    prm = meshless.PARAMETERS(solver_type="sor", solver_tolerance=1e-10)
    prm.rho, prm.mu, prm.dt = 1.0, 0.01, 2e-4
    pts = meshless.POINTS(cl)
    cld = meshless.CLOUD(pts, prm, compute_cond=False)
    fs = meshless.FRACTIONAL_STEP_1(pts, cld, prm, cl.u_dirichlet, cl.v_dirichlet,
                                    cl.p_dirichlet, 2)
    assert "solver_type sor" in capsys.readouterr().out
    fs.set_state([cl.vel_bc[0], cl.vel_bc[1]], np.zeros(fs.system_size), 0)
    fs.step(2)
    assert fs.last_stats()[1] <= 1e-10
    # the C entry point itself refuses SOR inside an integrator
    import ctypes as C
    flags = [np.ascontiguousarray(f, np.uint8) for f in (cl.u_dirichlet, cl.v_dirichlet,
                                                         cl.p_dirichlet)]
    cfg = prm.solver_cfg()
    assert cfg.precond == capi.MP_PRECOND_SOR
    h = C.c_void_p()
    rc = capi.lib().mp_fs1_create(cld.handle, ptr(pts.boundary_flag), ptr(pts.normal),
                                  ptr(flags[0]), ptr(flags[1]), None, ptr(flags[2]),
                                  C.byref(fs.cfg), C.byref(cfg), C.byref(h))
    assert rc == capi.MP_BAD_ARG and "sor" in capi.last_error()
