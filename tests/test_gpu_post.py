"""GPU: the restart reader's nearest-node lookup and the residual diagnostics."""
import numpy as np
import pytest
import scipy.sparse as sp

from memphys_b200 import capi, clouds, meshless, post

pytestmark = pytest.mark.gpu


def cavity(nx=24, reorder=None):
    cl = clouds.cavity_2d(nx, seed=7)
    prm = meshless.PARAMETERS(solver_type="cuda_bicgstab_amg")
    prm.rho, prm.mu = 1.0, 0.01
    pts = meshless.POINTS(cl)
    cld = meshless.CLOUD(pts, prm, compute_cond=False, reorder=reorder).fetch()
    return cl, prm, pts, cld


def test_restart_round_trip(mp_lib, tmp_path):
    cl, prm, pts, cld = cavity()
    x, y = pts.xyz[:, 0], pts.xyz[:, 1]
    u, p = np.sin(3 * x) * y, np.cos(2 * y) + x / 3.0
    prefix = str(tmp_path / "run")
    path = post.write_tecplot_steady_variables(prefix, pts, ["u", "p"], [u, p])
    ru, rp = post.read_restart_tecplot_file(pts, path, ["u", "p"])   # "p" is the last column
    assert np.allclose(ru, u, rtol=1e-15, atol=1e-15) and np.allclose(rp, p, rtol=1e-15, atol=1e-15)
    # a renumbered cloud of the same nodes reads the same values at its own numbering
    _, _, pts2, _ = cavity(reorder="rcm")
    (u2,) = post.read_restart_tecplot_file(pts2, path, ["u"])
    assert np.allclose(u2[pts2.order], u, rtol=1e-15, atol=1e-15)
    with pytest.raises(capi.MemphysError):
        post.read_restart_tecplot_file(pts, path, ["w"])


def test_knn_probe_nearest(mp_lib):
    cl = clouds.cavity_2d(20, seed=2)
    probe = np.random.default_rng(1).uniform(-0.1, 1.1, size=(500, 2))
    cols = np.zeros((500, 3), np.int32)
    capi.check(capi.lib().mp_knn_probe(capi.ptr(cl.xyz), cl.nv, 2, capi.ptr(probe), 500, 3,
                                       capi.ptr(cols), None))
    d2 = ((probe[:, None, :] - cl.xyz[None, :, :]) ** 2).sum(2)
    ref = np.argsort(d2, axis=1, kind="stable")[:, :3]
    assert np.array_equal(cols, ref)


def test_navier_stokes_residuals(mp_lib):
    cl, prm, pts, cld = cavity()
    x, y = pts.xyz[:, 0], pts.xyz[:, 1]
    u, v, p = np.sin(x) * np.cos(y), -np.cos(x) * np.sin(y), x * y
    out = post.calc_navier_stokes_residuals_2D(pts, cld, prm, u, v, np.append(p, 0.0))
    rows = np.repeat(np.arange(cl.nv), cld.n)
    mk = lambda w: sp.csr_matrix((w.ravel(), (rows, cld.nb_points_col.ravel())), (cl.nv, cl.nv))
    Gx, Gy, L = mk(cld.grad_x_coeff), mk(cld.grad_y_coeff), mk(cld.laplacian_coeff)
    xm = u * (Gx @ u) + v * (Gy @ u) - 0.01 * (L @ u) + Gx @ p
    assert np.isclose(out["x_momentum"]["overall"][0], np.abs(xm).max(), rtol=1e-12)
    assert np.isclose(out["x_momentum"]["overall"][1], np.abs(xm).mean(), rtol=1e-12)
    b = pts.boundary_flag.astype(bool)
    cont = Gx @ u + Gy @ v
    assert np.isclose(out["continuity"]["internal"][0], np.abs(cont[~b]).max(), rtol=1e-12)
    # the divergence-free field: interior continuity residual is the stencils' truncation error
    assert out["continuity"]["internal"][0] < 1e-3
