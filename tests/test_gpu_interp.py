"""GPU: the interpolation matrix (mp_interp_matrix) against its oracle.

calc_interp_matrix (coefficient_computations.cpp:456-518): each probe's n
nearest nodes and the PHS r^3 + degree-3 interpolation weights.  Columns must
equal the oracle's exactly (integer), weights to a relative 1e-9 per row, and
the weights must reproduce cubic polynomials at the probes.
"""
import numpy as np
import pytest

import oracle
from memphys_b200 import capi, clouds
from memphys_b200.capi import ptr

pytestmark = pytest.mark.gpu


def interp(xyz, probe, n, phs=3, poly=3):
    npb = len(probe)
    cols = np.zeros((npb, n), np.int32)
    w = np.zeros((npb, n))
    capi.check(capi.lib().mp_interp_matrix(ptr(np.ascontiguousarray(xyz)), len(xyz), xyz.shape[1],
                                           ptr(np.ascontiguousarray(probe)), npb, n, phs, poly,
                                           ptr(cols), ptr(w), None), "mp_interp_matrix")
    return cols, w


@pytest.mark.parametrize("make,n,np_", [(lambda: clouds.cavity_2d(30, seed=2), 20, 300),
                                        (lambda: clouds.cube_3d(8, seed=3), 40, 200)])
def test_interp_matches_oracle_and_reproduces_cubics(mp_lib, make, n, np_):
    cl = make()
    rng = np.random.default_rng(5)
    dim = cl.dim
    probe = rng.uniform(0.02, 0.98, size=(np_, dim))
    probe[:5] = cl.xyz[[3, 17, 40, 77, 101]]          # probes on nodes: interpolation is exact
    probe[5] = [1.03] + [0.5] * (dim - 1)               # outside the cloud's box
    cols, w = interp(cl.xyz, probe, n)
    rc, rw = oracle.interp_matrix(cl.xyz, probe, n)
    assert np.array_equal(cols, rc)
    scale = np.abs(rw).max(1, keepdims=True)
    assert np.all(np.abs(w - rw) <= 1e-9 * scale)
    x = cl.xyz
    f = x[:, 0] ** 3 - 2 * x[:, 1] ** 2 * x[:, 0] + 0.5 * x[:, -1] + 3.0
    fp = probe[:, 0] ** 3 - 2 * probe[:, 1] ** 2 * probe[:, 0] + 0.5 * probe[:, -1] + 3.0
    assert np.abs((w * f[cols]).sum(1) - fp).max() <= 1e-9
    for k in range(5):  # a probe on node j gets weight 1 on j
        j = [3, 17, 40, 77, 101][k]
        assert abs(w[k][cols[k] == j][0] - 1.0) <= 1e-9


@pytest.mark.parametrize("n,poly", [(40, 1), (39, 1), (33, 3)])
def test_interp_largest_systems_of_a_class(mp_lib, n, poly):
    """Interpolation systems have one right-hand side, so a register-width class holds
    up to W - 1 rows (here n + m = 42-43 in the 44-wide class), two more than a
    weights system of the same class: every elimination step and every stencil point
    must still be there (the oracle solves the same systems with LAPACK)."""
    cl = clouds.cavity_2d(30, seed=4)
    rng = np.random.default_rng(11)
    probe = rng.uniform(0.05, 0.95, size=(200, 2))
    cols, w = interp(cl.xyz, probe, n, poly=poly)
    rc, rw = oracle.interp_matrix(cl.xyz, probe, n, poly_deg=poly)
    assert np.array_equal(cols, rc)
    scale = np.abs(rw).max(1, keepdims=True)
    assert np.all(np.abs(w - rw) <= 1e-9 * scale)
    assert np.abs(w.sum(1) - 1.0).max() <= 1e-9  # constants are reproduced


def test_interp_rejects_bad_arguments(mp_lib):
    cl = clouds.cavity_2d(10, seed=1)
    probe = np.array([[0.5, 0.5]])
    cols = np.zeros((1, 20), np.int32)
    w = np.zeros((1, 20))
    L = capi.lib()
    assert L.mp_interp_matrix(ptr(cl.xyz), cl.nv, 2, ptr(probe), 1, 70, 3, 3, ptr(cols), ptr(w),
                              None) == capi.MP_BAD_ARG
    assert L.mp_interp_matrix(ptr(cl.xyz), cl.nv, 2, ptr(probe), 1, 20, 4, 3, ptr(cols), ptr(w),
                              None) == capi.MP_BAD_ARG
