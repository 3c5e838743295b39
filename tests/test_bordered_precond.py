"""The bordered pressure system's preconditioner: its algebra, checked on the CPU.

An all-Neumann pressure system is bordered as solver.cpp:205-213 does it,
B = [A e; e^T 0] with e = ones and A e = 0.  The multigrid preconditioner the GPU
applies to it (mp_krylov.cu, Defl) is

    M^-1 [r; r_n] = [V(r - a e) + c e; a],   a = w^T r / w^T e,   c = (r_n - e^T V(r - a e)) / n

with V the multigrid cycle and w the weights of the mean: 1 on interior rows and
beta on boundary rows, beta fitted at set-up so that w^T A f = 0 for f = |x|^2.
On the oracle's operator of small cavities: with V a generalized inverse of A and
w the left null vector of A, M^-1 is exactly B's inverse; with the plain mean
(w = e) B M^-1 is the identity up to a rank-one term; the fitted weights follow
the left null vector (Green's identity: volume shares inside, minus surface
shares on the boundary).
"""
import numpy as np
import scipy.linalg as la

import oracle
from memphys_b200 import clouds


def bordered_operator(nx):
    cl = clouds.cavity_2d(nx, seed=2)
    nb = oracle.knn_stencils(cl.xyz, cl.boundary.astype(np.uint8), 20)
    w = oracle.cloud_weights(cl.xyz, nb, 3, 3, cond=False)
    rp, ci, val, ns = oracle.ppe_assemble(nb, w, cl.boundary, np.zeros(cl.nv, bool), cl.normal)
    B = np.zeros((ns, ns))
    for i in range(ns):
        np.add.at(B[i], ci[rp[i]:rp[i + 1]], val[rp[i]:rp[i + 1]])
    return cl, B


def fitted_weights(cl, A):
    f = (cl.xyz ** 2).sum(1)
    af = A @ f
    b = cl.boundary
    beta = -af[~b].sum() / af[b].sum()
    return np.where(b, beta, 1.0)


def preconditioner(G, w, n):
    """M^-1 as a dense matrix, column by column."""
    e = np.ones(n)
    M = np.zeros((n + 1, n + 1))
    for k in range(n + 1):
        r, rn = np.zeros(n), 0.0
        if k < n:
            r[k] = 1.0
        else:
            rn = 1.0
        a = w @ r / (w @ e)
        z = G @ (r - a * e)
        c = (rn - e @ z) / n
        M[:n, k] = z + c * e
        M[n, k] = a
    return M


def test_exact_with_the_left_null_vector_rank_one_with_the_plain_mean():
    cl, B = bordered_operator(12)
    n = cl.nv
    assert B.shape == (n + 1, n + 1)
    assert np.all(B[:n, n] == 1.0) and np.all(B[n, :n] == 1.0)
    A = B[:n, :n]
    assert np.abs(A.sum(1)).max() <= 1e-12 * np.abs(A).max()     # A e = 0 to rounding
    ell = la.null_space(A.T, rcond=1e-10)
    assert ell.shape[1] == 1
    ell = ell[:, 0]
    G = np.linalg.pinv(A, rcond=1e-10)                            # a generalized inverse
    I = np.eye(n + 1)
    exact = B @ preconditioner(G, ell, n) - I
    assert np.abs(exact).max() <= 1e-8
    s = np.linalg.svd(B @ preconditioner(G, np.ones(n), n) - I, compute_uv=False)
    assert s[0] > 1e-3 and s[1] <= 1e-8 * s[0]                   # one direction left


def test_fitted_weights_follow_the_left_null_vector():
    cl, B = bordered_operator(24)
    n = cl.nv
    A = B[:n, :n]
    ell = la.null_space(A.T, rcond=1e-10)[:, 0]
    b = cl.boundary
    ell = ell / ell[~b].mean()
    w = fitted_weights(cl, A)
    # interior 1, boundary about -1/h: the exact vector's boundary / interior ratio
    ratio_exact, ratio_fit = ell[b].mean(), w[b].mean()
    assert ratio_fit < 0 and abs(ratio_fit - ratio_exact) <= 0.02 * abs(ratio_exact)
    assert abs(ratio_exact * (1.0 / 24) + 1.0) <= 0.1             # about -1/h, h = 1/24
    # a vector in A's range has no weighted mean (the null vector is orthogonal to the
    # range); the plain mean sees part of it
    x, y = cl.xyz[:, 0], cl.xyz[:, 1]
    r = A @ (x ** 2 * y + 0.5 * y ** 3)
    print("weighted / plain mean of a range vector:", abs(w @ r) / abs(w @ np.ones(n)),
          abs(r.mean()))
    assert abs(w @ r) / abs(w @ np.ones(n)) <= 0.05 * abs(r.mean())
