"""GPU: the Fourier-z fractional step (mp_fsf_*) against its oracle.

FRACTIONAL_STEP_FOURIER restated in oracle/fsf.py on the reference's full
complex coefficient matrices with direct per-mode solves; the GPU stores the
modes 0..nw and solves each mode's Helmholtz system by BiCGSTAB + multigrid.
Two periods, so that the reference's DFT matrices (their phase carries the
period) are followed as written; full-Neumann pressure (bordered first mode).
"""
import numpy as np
import pytest

import oracle
from oracle import fsf as ofsf
from memphys_b200 import clouds, meshless

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("period", [1.0, 1.7])
def test_fsf_matches_oracle(mp_lib, period):
    cl = clouds.cavity_2d(16, seed=5)
    nw = 2
    N = 2 * nw + 1
    # 1e-9: the shifted Helmholtz systems floor near 6e-10 in FP64 on this cloud
    prm = meshless.PARAMETERS(solver_type="cuda_bicgstab_amg", solver_tolerance=1e-9, n_iter=5000)
    prm.rho, prm.mu, prm.dt = 1.0, 0.01, 1e-3
    pts = meshless.POINTS(cl)
    cld = meshless.CLOUD(pts, prm, compute_cond=False).fetch()
    fs = meshless.FRACTIONAL_STEP_FOURIER(pts, cld, prm, cl.u_dirichlet, cl.v_dirichlet,
                                          cl.u_dirichlet, cl.p_dirichlet, period, nw, 2)
    w = {"gx": cld.grad_x_coeff, "gy": cld.grad_y_coeff, "lap": cld.laplacian_coeff}
    ref = ofsf.FSF(cl, cld.nb_points_col, w, 1.0, 0.01, 1e-3, cl.u_dirichlet, cl.v_dirichlet,
                   cl.u_dirichlet, cl.p_dirichlet, period, nw)
    z = np.arange(N) * period / N
    x, y = cl.xyz[:, 0], cl.xyz[:, 1]
    u = np.repeat(cl.vel_bc[0][:, None], N, 1)
    v = np.zeros((cl.nv, N))
    wz = np.where(cl.boundary[:, None], 0.0,
                  0.05 * (np.sin(np.pi * x) * np.sin(np.pi * y))[:, None]
                  * np.cos(2 * np.pi * z / period)[None, :])
    p = np.zeros((cl.nv, N))
    g = [a.copy() for a in (u, v, wz, p)]
    r = [a.copy() for a in (u, v, wz, p)]
    for it in range(4):
        out = [np.zeros((cl.nv, N)) for _ in range(4)]
        fs.single_timestep(*out, *g, it)
        g = out
        r = list(ref.single_timestep(*r, it))
    for name, a, b in zip("uvwp", g, r):
        scale = max(np.abs(b).max(), 1e-12)
        print(name, np.abs(a - b).max() / scale)
        assert np.abs(a - b).max() <= 1e-7 * scale, name
    assert np.abs(g[2]).max() > 1e-3          # the z-dependent part survives the steps


def test_fsf_layouts_agree(mp_lib):
    """The two field layouts of mp_fsf_single_timestep: plane-contiguous (Eigen's
    column-major, host arrays straight through the C ABI) and node-major (numpy's
    C-ordered (nv, N), transposed on the device, the Python mirror's) give the same
    fields bit for bit; an unknown layout is refused."""
    import ctypes as C
    from memphys_b200 import capi
    cl = clouds.cavity_2d(16, seed=5)
    nw, N = 2, 5
    prm = meshless.PARAMETERS(solver_type="cuda_bicgstab_amg", solver_tolerance=1e-9, n_iter=5000)
    prm.rho, prm.mu, prm.dt = 1.0, 0.01, 1e-3
    pts = meshless.POINTS(cl)
    cld = meshless.CLOUD(pts, prm, compute_cond=False)
    make = lambda: meshless.FRACTIONAL_STEP_FOURIER(pts, cld, prm, cl.u_dirichlet, cl.v_dirichlet,
                                                    cl.u_dirichlet, cl.p_dirichlet, 1.0, nw, 2)
    a, b = make(), make()
    L = capi.lib()
    assert L.mp_fsf_set_layout(b.handle, 2) == capi.MP_BAD_ARG
    capi.check(L.mp_fsf_set_layout(b.handle, 0))
    z = np.arange(N) / N
    x, y = cl.xyz[:, 0], cl.xyz[:, 1]
    g = [np.repeat(cl.vel_bc[0][:, None], N, 1), np.zeros((cl.nv, N)),
         np.where(cl.boundary[:, None], 0.0,
                  0.05 * (np.sin(np.pi * x) * np.sin(np.pi * y))[:, None]
                  * np.cos(2 * np.pi * z)[None, :]), np.zeros((cl.nv, N))]
    ga = [q.copy() for q in g]
    gb = [np.ascontiguousarray(q.T) for q in g]     # (N, nv): plane c contiguous
    for it in range(3):
        oa = [np.zeros((cl.nv, N)) for _ in range(4)]
        a.single_timestep(*oa, *ga, it)
        ga = oa
        ob = [np.zeros((N, cl.nv)) for _ in range(4)]
        vin = (C.c_void_p * 3)(*[q.ctypes.data for q in gb[:3]])
        vout = (C.c_void_p * 3)(*[q.ctypes.data for q in ob[:3]])
        capi.check(L.mp_fsf_single_timestep(b.handle, vin, capi.ptr(gb[3]), vout,
                                            capi.ptr(ob[3]), it, None))
        gb = ob
    for name, qa, qb in zip("uvwp", ga, gb):
        assert np.array_equal(qa, qb.T), name
