"""GPU: node orderings (mp_order_rcm, mp_order_morton) and reordered clouds.

The reference's CLOUD constructor renumbers every cloud by reverse
Cuthill-McKee on the stencil graph (cloud.cpp:37, general_functions.cpp:806-879)
and permutes points and stencils (re_order_points, cloud.cpp:337-439).  The
RCM order must equal the oracle's restatement exactly; the Morton order must be
a permutation that sorts the quantised Z-order codes; a reordered cloud must
carry the same weights (bit for bit, permuted) and give the same flow.
"""
import numpy as np
import pytest

import oracle
from memphys_b200 import capi, clouds, meshless
from memphys_b200.capi import ptr

pytestmark = pytest.mark.gpu


def knn(cl, n):
    nb = np.zeros((cl.nv, n), np.int32)
    capi.check(capi.lib().mp_knn_stencils(ptr(cl.xyz), ptr(cl.boundary), cl.nv, cl.dim, n,
                                          ptr(nb), None), "mp_knn_stencils")
    return nb


@pytest.mark.parametrize("make,n", [(lambda: clouds.cavity_2d(40, seed=2), 20),
                                    (lambda: clouds.cube_3d(9, seed=4), 40),
                                    (lambda: clouds.channel_2d(0.05, seed=3), 20)])
def test_rcm_matches_reference_algorithm(mp_lib, make, n):
    cl = make()
    nb = knn(cl, n)
    order = np.zeros(cl.nv, np.int32)
    capi.check(capi.lib().mp_order_rcm(ptr(nb), cl.nv, n, ptr(order)), "mp_order_rcm")
    assert np.array_equal(order, oracle.rcm_order(nb))
    assert np.array_equal(np.sort(order), np.arange(cl.nv))


def morton_codes(xyz):
    dim = xyz.shape[1]
    bits = 21 if dim == 3 else 16
    cells = float((1 << bits) - 1)
    lo, hi = xyz.min(0), xyz.max(0)
    t = (xyz - lo) / np.where(hi > lo, hi - lo, 1.0)
    q = np.clip(np.floor(t * cells), 0, cells).astype(np.uint64)
    code = np.zeros(len(xyz), np.uint64)
    for b in range(bits):
        for d in range(dim):
            code |= ((q[:, d] >> np.uint64(b)) & np.uint64(1)) << np.uint64(dim * b + d)
    return code


@pytest.mark.parametrize("make", [lambda: clouds.cavity_2d(50, seed=5),
                                  lambda: clouds.cube_3d(10, seed=6)])
def test_morton_order_sorts_codes(mp_lib, make):
    cl = make()
    order = np.zeros(cl.nv, np.int32)
    capi.check(capi.lib().mp_order_morton(ptr(cl.xyz), cl.nv, cl.dim, ptr(order), None),
               "mp_order_morton")
    assert np.array_equal(np.sort(order), np.arange(cl.nv))
    inv = np.empty_like(order)
    inv[order] = np.arange(cl.nv)          # inv[r] = node at rank r
    code = morton_codes(cl.xyz)[inv]
    assert np.all(code[1:] >= code[:-1])
    ties = code[1:] == code[:-1]
    assert np.all(inv[1:][ties] > inv[:-1][ties])   # equal codes keep index order


def test_permute_stencils_and_rows(mp_lib):
    cl = clouds.cavity_2d(30, seed=1)
    nb = knn(cl, 20)
    order = np.random.default_rng(0).permutation(cl.nv).astype(np.int32)
    out = np.zeros_like(nb)
    capi.check(capi.lib().mp_permute_stencils(ptr(nb), cl.nv, 20, ptr(order), ptr(out), None))
    assert np.array_equal(out[order], order[nb])
    xyz = np.ascontiguousarray(cl.xyz)
    moved = np.empty_like(xyz)
    capi.check(capi.lib().mp_permute_rows(ptr(xyz), ptr(moved), cl.nv, 16, ptr(order), None))
    assert np.array_equal(moved[order], xyz)
    bad = nb.copy()
    bad[3, 4] = cl.nv
    assert capi.lib().mp_permute_stencils(ptr(bad), cl.nv, 20, ptr(order), ptr(out),
                                          None) == capi.MP_BAD_ARG


@pytest.mark.parametrize("reorder", ["rcm", "morton"])
def test_reordered_cloud_same_weights_and_flow(mp_lib, reorder):
    cl = clouds.cavity_2d(32, seed=3)
    prm = meshless.PARAMETERS(solver_type="cuda_bicgstab_amg", solver_tolerance=1e-11,
                              n_iter=5000)
    prm.rho, prm.mu, prm.dt = 1.0, 0.01, 2e-4
    base_pts = meshless.POINTS(cl)
    base = meshless.CLOUD(base_pts, prm, compute_cond=False).fetch()
    pts = meshless.POINTS(cl)
    cld = meshless.CLOUD(pts, prm, compute_cond=False, reorder=reorder).fetch()
    o = pts.order
    assert np.array_equal(pts.xyz[o], base_pts.xyz)
    assert np.array_equal(cld.nb_points_col[o], o[base.nb_points_col])
    for k in ("grad_x_coeff", "grad_y_coeff", "laplacian_coeff"):
        assert np.array_equal(getattr(cld, k)[o], getattr(base, k))   # same arithmetic per stencil
    res = []
    for P, C_ in ((base_pts, base), (pts, cld)):
        fs = meshless.FRACTIONAL_STEP_1(P, C_, prm, P.permute(cl.u_dirichlet),
                                        P.permute(cl.v_dirichlet), P.permute(cl.p_dirichlet), 2)
        fs.set_state([P.permute(cl.vel_bc[0]), P.permute(cl.vel_bc[1])],
                     np.zeros(fs.system_size), 0)
        fs.step(6)
        vel, p = fs.get_state()
        res.append((vel, p[:cl.nv], fs.log(0, 6)))
    (v0, p0, l0), (v1, p1, l1) = res
    for d in range(2):
        assert np.abs(v1[d][o] - v0[d]).max() <= 1e-7 * np.abs(v0[d]).max()
    assert np.all(l1[:, 1] <= 1e-11)
