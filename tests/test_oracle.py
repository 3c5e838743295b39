"""CPU oracle pinned against the reference's own outputs (no GPU needed).

Pins:
  - sample_stats.json: the reference's sample-run statistics
    (Sample outputs/..._simulation_details.csv) for the shipped annulus mesh:
    node counts, dx statistics, RBF condition numbers, largest eigenvalues.
  - ecc_cloud.npz / knn_cavity.npz: stencils from the reference's vendored
    nanoflann (oracle/ref_knn.cpp).
  - lapack_stencils.npz: per-stencil weights from LAPACK dgesv.
"""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as sla

import oracle
from oracle import fs1 as ofs1
from oracle import msh
from memphys_b200 import clouds


@pytest.fixture(scope="module")
def ecc(golden_dir):
    g = np.load(os.path.join(golden_dir, "ecc_cloud.npz"))
    stats = json.load(open(os.path.join(golden_dir, "sample_stats.json")))
    nb = oracle.knn_stencils(g["xyz"], g["boundary"], stats["cloud_size"])
    w = oracle.cloud_weights(g["xyz"], nb, stats["phs_deg"], stats["poly_deg"])
    return g, stats, nb, w


def test_poly_exponents_order():
    # parameters.cpp:217-267
    e2 = oracle.poly_exponents(2, 3).tolist()
    assert e2 == [[0, 0], [1, 0], [0, 1], [2, 0], [1, 1], [0, 2], [3, 0], [2, 1], [1, 2], [0, 3]]
    e3 = oracle.poly_exponents(3, 3).tolist()
    assert e3[:4] == [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]]
    assert e3[4:10] == [[2, 0, 0], [1, 1, 0], [1, 0, 1], [0, 2, 0], [0, 1, 1], [0, 0, 2]]
    assert e3[10:] == [[3, 0, 0], [2, 1, 0], [2, 0, 1], [1, 2, 0], [1, 1, 1], [1, 0, 2],
                       [0, 3, 0], [0, 2, 1], [0, 1, 2], [0, 0, 3]]
    for dim in (2, 3):
        for p in range(2, 9):
            e = oracle.poly_exponents(dim, p)
            assert len({tuple(r) for r in e.tolist()}) == e.shape[0]
            assert e.sum(1).max() == p
    assert oracle.cloud_size(2, 3, 2.0) == 20 and oracle.cloud_size(3, 3, 2.0) == 40


def test_sample_counts(ecc):
    g, stats, nb, w = ecc
    assert g["xyz"].shape[0] == stats["nv"]
    assert int(g["boundary"].sum()) == stats["nv_boundary"]


def test_sample_dx(ecc):
    g, stats, nb, w = ecc
    mx, mn, avg = msh.charac_dx(g["xyz"], nb)
    assert mx == pytest.approx(stats["dx_max"], rel=1e-12)
    assert mn == pytest.approx(stats["dx_min"], rel=1e-12)
    assert avg == pytest.approx(stats["dx_avg"], rel=1e-12)


def test_sample_condition_numbers(ecc):
    # coefficient_computations.cpp:312 (Eigen rcond estimate); cloud.cpp:273-276
    g, stats, nb, w = ecc
    ce = w["cond_est"]
    assert ce.max() == pytest.approx(stats["cond_max"], rel=1e-9)
    assert ce.min() == pytest.approx(stats["cond_min"], rel=1e-9)
    assert ce.mean() == pytest.approx(stats["cond_avg"], rel=1e-9)
    # the estimate never exceeds the exact 1-norm condition number
    assert np.all(ce <= w["cond_exact"] * (1 + 1e-10))


@pytest.mark.parametrize("key,name", [("gx", "grad_x_eig"), ("gy", "grad_y_eig"),
                                      ("lap", "laplace_eig")])
def test_sample_eigenvalues(ecc, key, name):
    # parameters.cpp:269-296 / general_functions.cpp:4-24 (largest-|lambda| Arnoldi)
    g, stats, nb, w = ecc
    nv = nb.shape[0]
    A = sp.csr_matrix((w[key].ravel(), (np.repeat(np.arange(nv), nb.shape[1]), nb.ravel())),
                      shape=(nv, nv))
    ev = sla.eigs(A, k=1, which="LM", ncv=20, return_eigenvectors=False)[0]
    re, im = stats[name]
    assert ev.real == pytest.approx(re, rel=1e-7)
    assert abs(ev.imag) == pytest.approx(abs(im), abs=1e-6 * abs(re))


def test_knn_matches_nanoflann(golden_dir):
    c = np.load(os.path.join(golden_dir, "knn_cavity.npz"))
    nb = oracle.knn_stencils(c["xyz"], c["boundary"], 20)
    assert np.array_equal(nb, c["nb_col_nanoflann"])
    g = np.load(os.path.join(golden_dir, "ecc_cloud.npz"))
    nb = oracle.knn_stencils(g["xyz"], g["boundary"], 20)
    ref = g["nb_col_nanoflann"]
    # same sets (the structured annulus has exact distance ties)
    assert all(set(a) == set(b) for a, b in zip(nb.tolist(), ref.tolist()))
    assert (nb != ref).sum() <= 4


def test_boundary_stencil_rule(golden_dir):
    # cloud.cpp:624-640: boundary node = itself + interior nodes only
    c = np.load(os.path.join(golden_dir, "knn_cavity.npz"))
    nb = oracle.knn_stencils(c["xyz"], c["boundary"], 20)
    b = c["boundary"]
    assert np.all(nb[:, 0] == np.arange(len(b)))
    assert not np.any(b[nb[b][:, 1:]])


@pytest.mark.parametrize("dim", [2, 3])
def test_weights_match_lapack(golden_dir, dim):
    L = np.load(os.path.join(golden_dir, "lapack_stencils.npz"))
    sizes = L[f"sizes{dim}"]
    off = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    w, _, bad = oracle.batched_weights(sizes, off, L[f"pts{dim}"], dim)
    assert bad == 0
    ref = L[f"w{dim}"]
    for n, o in zip(sizes, off):
        a = w[(dim + 1) * o:(dim + 1) * (o + n)]
        b = ref[(dim + 1) * o:(dim + 1) * (o + n)]
        assert np.abs(a - b).max() <= 1e-8 * np.abs(b).max()


@pytest.mark.parametrize("dim", [2, 3])
def test_polynomial_reproduction(dim):
    # constraint rows of A (coefficient_computations.cpp:90-102): sum_j w_ij q(x_j)
    # equals the derivative of q at x_i for every monomial of degree <= 3
    cl = clouds.cavity_2d(12) if dim == 2 else clouds.cube_3d(6)
    n = oracle.cloud_size(dim, 3, 2.0)
    nb = oracle.knn_stencils(cl.xyz, cl.boundary, n)
    w = oracle.cloud_weights(cl.xyz, nb, 3, 3, cond=False)
    e = oracle.poly_exponents(dim, 3)
    x = cl.xyz
    for ex in e:
        q = np.prod(x ** ex, axis=1)
        for k, key in enumerate(["gx", "gy", "gz"][:dim]):
            d = np.zeros(len(x))
            if ex[k] > 0:
                ee = ex.copy()
                ee[k] -= 1
                d = ex[k] * np.prod(x ** ee, axis=1)
            got = (w[key] * q[nb]).sum(1)
            assert np.abs(got - d).max() <= 1e-6 * max(1.0, np.abs(d).max())
        lap = np.zeros(len(x))
        for k in range(dim):
            if ex[k] > 1:
                ee = ex.copy()
                ee[k] -= 2
                lap += ex[k] * (ex[k] - 1) * np.prod(x ** ee, axis=1)
        got = (w["lap"] * q[nb]).sum(1)
        assert np.abs(got - lap).max() <= 1e-4 * max(1.0, np.abs(lap).max())


def test_ppe_assembly_structure():
    # solver.cpp:165-214: Neumann rows n.grad, bordered with ones, (nv,nv) = 0
    cl = clouds.cavity_2d(10)
    nb = oracle.knn_stencils(cl.xyz, cl.boundary, 20)
    w = oracle.cloud_weights(cl.xyz, nb, 3, 3, cond=False)
    rp, ci, val, ns = oracle.ppe_assemble(nb, w, cl.boundary, cl.p_dirichlet, cl.normal)
    nv = cl.nv
    assert ns == nv + 1
    A = sp.csr_matrix((val, ci, rp), shape=(ns, ns)).toarray()
    assert np.all(A[nv, :nv] == 1.0) and A[nv, nv] == 0.0 and np.all(A[:nv, nv] == 1.0)
    # constants are in the kernel of the stencil part (rows sum to zero)
    assert np.abs(A[:nv, :nv].sum(1)).max() < 1e-6 * np.abs(A[:nv, :nv]).max()
    i = np.nonzero(cl.boundary)[0][0]
    expect = cl.normal[i, 0] * w["gx"][i] + cl.normal[i, 1] * w["gy"][i]
    assert np.allclose(A[i, nb[i]], expect)
    # a Dirichlet node removes the border (solver.cpp:33-38)
    pd = cl.p_dirichlet.copy()
    pd[i] = True
    rp2, ci2, val2, ns2 = oracle.ppe_assemble(nb, w, cl.boundary, pd, cl.normal)
    assert ns2 == nv and rp2[i + 1] - rp2[i] == 1 and val2[rp2[i]] == 1.0


def test_bicgstab_converges_to_direct_solution():
    cl = clouds.cavity_2d(20)
    nb = oracle.knn_stencils(cl.xyz, cl.boundary, 20)
    w = oracle.cloud_weights(cl.xyz, nb, 3, 3, cond=False)
    rp, ci, val, ns = oracle.ppe_assemble(nb, w, cl.boundary, cl.p_dirichlet, cl.normal)
    A = sp.csr_matrix((val, ci, rp), shape=(ns, ns))
    b = np.random.default_rng(3).standard_normal(ns)
    b[-1] = 0.0
    xd = sla.spsolve(A.tocsc(), b)
    f = oracle.ILUT(rp, ci, val, 1e-6, 50)
    x, it, rr, rec = oracle.bicgstab(rp, ci, val, b, tol=1e-10, maxit=2000, precond=f)
    assert rr <= 1e-9
    assert np.abs(x - xd).max() <= 1e-6 * np.abs(xd).max()


def test_fs1_oracles_agree():
    # the C restatement (BiCGSTAB + ILUT) and the numpy one (direct LU) give the
    # same fields to the solver tolerance
    cl = clouds.cavity_2d(16)
    nb = oracle.knn_stencils(cl.xyz, cl.boundary, 20)
    w = oracle.cloud_weights(cl.xyz, nb, 3, 3, cond=False)
    dt = 2e-4
    a = oracle.FS1(cl, nb, w, 1.0, 0.01, dt, 2, 1e-12, 2000, 1e-6, 50)
    b = ofs1.FS1(cl, nb, w, 1.0, 0.01, dt, 2)
    va = [cl.vel_bc[0].copy(), cl.vel_bc[1].copy()]
    vb = [cl.vel_bc[0].copy(), cl.vel_bc[1].copy()]
    pa, pb = np.zeros(a.nsys), np.zeros(b.nsys)
    for it in range(5):
        a.step(va, pa, it)
        b.step(vb, pb, it)
    for d in range(2):
        assert np.abs(va[d] - vb[d]).max() <= 1e-9 * np.abs(vb[d]).max()
    assert np.abs(pa - pb).max() <= 1e-7 * np.abs(pb).max()


def test_c1_configured_dt_is_unstable():
    """C1's configured dt = 1e-3 is above the explicit limit of the AB2 step on the
    100 x 100 jittered cavity: the largest-magnitude eigenvalues (ARPACK) are
    grad_x -388.9, grad_y 307.2 and laplacian -4.112e5, so calc_dt's rule
    (parameters.cpp:269-296) gives dt = Courant * 4.16e-4, and mu * dt * |lambda_L| =
    4.1 at dt = 1e-3 (AB2 needs < 1).  The oracle blows up within 10 steps there
    (|u| ~ 5e7 at step 6) and stays bounded over 50 steps at the calc_dt step of
    Courant 0.25 that the GPU tests and the benchmark use."""
    cl = clouds.cavity_2d(100)
    nb = oracle.knn_stencils(cl.xyz, cl.boundary, 20)
    w = oracle.cloud_weights(cl.xyz, nb, 3, 3, cond=False)
    nv = cl.nv
    rows = np.repeat(np.arange(nv), 20)
    lam = {}
    for k in ("gx", "gy", "lap"):
        A = sp.csr_matrix((w[k].ravel(), (rows, nb.ravel())), shape=(nv, nv))
        lam[k] = abs(sla.eigs(A, k=1, which="LM", ncv=30, return_eigenvectors=False)[0])
    assert lam["gx"] == pytest.approx(388.93, rel=1e-4)
    assert lam["lap"] == pytest.approx(4.1122e5, rel=1e-4)
    dt_calc = 0.25 * 2.0 / (lam["gx"] + lam["gy"] + 0.01 * lam["lap"])
    assert 0.01 * 1e-3 * lam["lap"] > 4.0
    for dt, nsteps, bounded in ((1e-3, 10, False), (dt_calc, 50, True)):
        f = ofs1.FS1(cl, nb, w, 1.0, 0.01, dt, 2)
        vel = [cl.vel_bc[0].copy(), cl.vel_bc[1].copy()]
        p = np.zeros(f.nsys)
        umax = 0.0
        for it in range(nsteps):
            f.step(vel, p, it)
            umax = max(umax, float(np.nan_to_num(np.abs(vel[0]).max(), nan=np.inf)))
        assert (umax <= 1.0 + 1e-9) == bounded, (dt, umax)


def test_oracle_threads_do_not_change_results():
    # the row-parallel loops (SpMV rows, fractional-step row loops) compute every
    # row as the serial loop does; dot products and ILUT solves stay serial
    cl = clouds.cavity_2d(64, seed=5)
    nb = oracle.knn_stencils(cl.xyz, cl.boundary, 20)
    w = oracle.cloud_weights(cl.xyz, nb, 3, 3, cond=False)
    out = []
    prev = oracle.set_threads(1)
    try:
        for threads in (1, 4):
            oracle.set_threads(threads)
            f = oracle.FS1(cl, nb, w, 1.0, 0.01, 1e-4, 2, 1e-8, 30, 1e-6, 50)
            vel = [cl.vel_bc[0].copy(), cl.vel_bc[1].copy()]
            p = np.zeros(f.nsys)
            for it in range(3):
                f.step(vel, p, it)
            out.append((vel[0], vel[1], p))
    finally:
        oracle.set_threads(prev)
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_fourier_transforms_as_the_reference_writes_them():
    # get_dft_matrix / get_idft_matrix (general_functions.cpp:1106-1123) divide the
    # phase by the period: the pair inverts for period 1 only, and the step follows
    # the matrices as written (the GPU path reproduces them for parity)
    from oracle import fsf as ofsf
    cl = clouds.cavity_2d(6, seed=1)
    nb = oracle.knn_stencils(cl.xyz, cl.boundary, 20)
    w = oracle.cloud_weights(cl.xyz, nb, 3, 3, cond=False)
    x = np.random.default_rng(0).standard_normal((cl.nv, 5))
    err = {}
    for period in (1.0, 1.7):
        f = ofsf.FSF(cl, nb, w, 1.0, 0.01, 1e-3, cl.u_dirichlet, cl.v_dirichlet,
                     cl.u_dirichlet, cl.p_dirichlet, period, 2)
        err[period] = np.abs(f.idft(f.dft(x)) - x).max()
    assert err[1.0] < 1e-14
    assert err[1.7] > 0.1


def test_sor_orders_converge_to_the_same_solution():
    """SOLVER::SOR (solver.cpp:243-281) in the reference's index order and in the
    multicolour order of the GPU sweeps: the colouring is proper (no row reads a row of
    its own colour), and on an implicit velocity-type system (rho/dt I - mu L inside,
    identity on the Dirichlet boundary, solver.cpp:165-204) both orders converge to the
    direct solution."""
    cl = clouds.cavity_2d(12, seed=2)
    nb = oracle.knn_stencils(cl.xyz, cl.boundary, 20)
    w = oracle.cloud_weights(cl.xyz, nb, 3, 3, cond=False)
    rp, ci, val, ns = oracle.ppe_assemble(nb, w, cl.boundary, cl.u_dirichlet, cl.normal,
                                          unsteady=2000.0, conv=0.0, diff=-1.0, bordered=False)
    assert ns == cl.nv
    colour = oracle.sor_colouring(rp, ci, val, ns)
    rows = np.repeat(np.arange(ns), np.diff(rp))
    off = ci != rows
    assert np.all(colour[rows[off]] != colour[ci[off]])
    A = sp.csr_matrix((val, ci, rp), shape=(ns, ns))
    b = np.random.default_rng(3).standard_normal(ns)
    xd = sla.spsolve(A.tocsc(), b)
    x_idx = oracle.sor_sweeps(rp, ci, val, b, np.zeros(ns), 1.4, 60)
    x_mc = oracle.sor_sweeps(rp, ci, val, b, np.zeros(ns), 1.4, 60, colour)
    for x in (x_idx, x_mc):
        assert np.linalg.norm(A @ x - b) <= 1e-10 * np.linalg.norm(b)
        assert np.abs(x - xd).max() <= 1e-10 * np.abs(xd).max()
    assert not np.allclose(oracle.sor_sweeps(rp, ci, val, b, np.zeros(ns), 1.4, 2),
                           oracle.sor_sweeps(rp, ci, val, b, np.zeros(ns), 1.4, 2, colour),
                           rtol=1e-6)  # the iterates themselves differ
