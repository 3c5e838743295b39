"""Failure detection through the C ABI (no GPU fault is ever provoked: the
failures are host-side argument errors or numerical conditions that the
kernels report as status codes)."""
import numpy as np
import pytest

from memphys_b200 import capi, clouds, meshless
from memphys_b200.capi import ptr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small(mp_lib):
    cl = clouds.cavity_2d(20, seed=1)
    pts = meshless.POINTS(cl)
    cld = meshless.CLOUD(pts, meshless.PARAMETERS(), compute_cond=False)
    return cl, pts, cld


def solver(small, **kw):
    cl, pts, cld = small
    p = meshless.PARAMETERS(**kw)
    return p, meshless.SOLVER().init(pts, cld, p, cl.p_dirichlet, 0.0, 0.0, 1.0, True)


def test_nan_rhs_reports_nan(small):
    p, s = solver(small)
    b = np.ones(s.system_size)
    b[3] = np.nan
    with pytest.raises(capi.MemphysError) as e:
        s.general_solve(small[1], p, np.zeros(s.system_size), np.zeros(s.system_size), b)
    assert e.value.status == capi.MP_NAN_DETECTED


def test_maxit_reports_not_converged(small):
    p, s = solver(small, n_iter=1, solver_type="cuda_bicgstab_jacobi")
    b = np.random.default_rng(0).standard_normal(s.system_size)
    b[-1] = 0
    x = np.zeros(s.system_size)
    with pytest.raises(capi.MemphysError) as e:
        s.general_solve(small[1], p, x, np.zeros(s.system_size), b)
    assert e.value.status == capi.MP_NOT_CONVERGED
    assert p.n_iter_actual[-1] == 1 and p.rel_res_log[-1] > 1e-8


def test_zero_rhs_gives_zero_solution(small):
    # Eigen's BiCGSTAB returns x = 0 when ||b|| = 0
    p, s = solver(small)
    x = np.zeros(s.system_size)
    s.general_solve(small[1], p, x, np.ones(s.system_size), np.zeros(s.system_size))
    assert np.all(x == 0.0)


def test_duplicate_nodes_are_singular(mp_lib):
    cl = clouds.cavity_2d(10, seed=1)
    xyz = cl.xyz.copy()
    xyz[5] = xyz[6]  # two nodes on top of each other
    nb = np.tile(np.arange(20, dtype=np.int32), (cl.nv, 1))
    nb[:, 0] = np.arange(cl.nv)
    nb[:20, :] = np.arange(20)
    w = [np.zeros((cl.nv, 20)) for _ in range(3)]
    rc = capi.lib().mp_stencil_weights(ptr(xyz), cl.nv, 2, ptr(nb), 20, 3, 3, ptr(w[0]),
                                       ptr(w[1]), None, ptr(w[2]), None, None)
    assert rc == capi.MP_SINGULAR_STENCIL
    assert "zero pivot" in capi.last_error()


@pytest.mark.parametrize("phs,poly,dim", [(4, 3, 2), (3, 1, 2), (3, 3, 4)])
def test_bad_parameters(mp_lib, phs, poly, dim):
    cl = clouds.cavity_2d(10)
    h = __import__("ctypes").c_void_p()
    bnd = cl.boundary.astype(np.uint8)
    rc = capi.lib().mp_cloud_create(ptr(cl.xyz), ptr(bnd), cl.nv, dim,
                                    phs, poly, 2.0, 0, None, __import__("ctypes").byref(h))
    assert rc == capi.MP_BAD_ARG


def test_knn_too_few_interior_nodes(mp_lib):
    xyz = np.random.default_rng(0).random((30, 2))
    bnd = np.ones(30, np.uint8)
    bnd[:5] = 0  # boundary nodes need n-1 = 19 interior neighbours
    out = np.zeros((30, 20), np.int32)
    rc = capi.lib().mp_knn_stencils(ptr(xyz), ptr(bnd), 30, 2, 20, ptr(out), None)
    assert rc == capi.MP_KNN_FAILED


def test_full_neumann_velocity_rejected(mp_lib):
    # fractional_step_1.cpp:80-91
    cl = clouds.cavity_2d(10)
    prm = meshless.PARAMETERS()
    prm.rho, prm.mu, prm.dt = 1.0, 0.01, 1e-4
    pts = meshless.POINTS(cl)
    cld = meshless.CLOUD(pts, prm, compute_cond=False)
    with pytest.raises(capi.MemphysError) as e:
        meshless.FRACTIONAL_STEP_1(pts, cld, prm, np.zeros(cl.nv, bool), cl.v_dirichlet,
                                   cl.p_dirichlet, 2)
    assert e.value.status == capi.MP_BAD_ARG and "full Neumann" in str(e.value)
