"""The synthetic point clouds every configuration is measured on (CPU).

No public dataset is involved: the clouds are jittered grids from a seeded
Philox stream.  These tests pin what the configurations state: the cavity's
nodes and boundary (100 x 100 interior nodes jittered by up to 0.2 h plus 100
boundary nodes per side without the corners, 10,400 in all; 1,004,000 at
1000 x 1000), the cube's n^3 interior nodes plus n^2 per face (2,195,456 at
128), the channel with its cylinder, unit outward normals on every boundary
node, the boundary conditions each carries, and reproducibility from the seed.
"""
import numpy as np
import pytest

from memphys_b200 import clouds


def test_cavity_nodes_boundary_and_conditions():
    nx = 100
    cl = clouds.cavity_2d(nx)
    h = 1.0 / nx
    assert cl.nv == 10_400 and cl.dim == 2
    ni = nx * nx
    assert not cl.boundary[:ni].any() and cl.boundary[ni:].all()
    # interior: each node within 0.2 h of its grid point, grid in row-major order
    c = (np.arange(nx) + 0.5) * h
    X, Y = np.meshgrid(c, c, indexing="xy")
    d = cl.xyz[:ni] - np.stack([X.ravel(), Y.ravel()], 1)
    assert np.abs(d).max() <= 0.2 * h and np.abs(d).max() > 0.19 * h
    # boundary: 100 per side on the walls, corners excluded
    b = cl.xyz[ni:]
    on_wall = np.isclose(b, 0.0) | np.isclose(b, 1.0)
    assert np.all(on_wall.sum(1) == 1)
    for axis in range(2):
        for v in (0.0, 1.0):
            assert np.isclose(b[:, axis], v).sum() == nx
    n = cl.normal[ni:]
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0)
    outward = np.where(np.isclose(b, 1.0), 1.0, np.where(np.isclose(b, 0.0), -1.0, 0.0))
    assert np.array_equal(n, outward)
    assert np.all(cl.normal[:ni] == 0.0)
    # Dirichlet velocity everywhere on the walls, the lid moving at 1, all-Neumann pressure
    assert np.array_equal(cl.u_dirichlet, cl.boundary) and np.array_equal(cl.v_dirichlet, cl.boundary)
    assert not cl.p_dirichlet.any()
    lid = cl.boundary & np.isclose(cl.xyz[:, 1], 1.0)
    assert np.all(cl.vel_bc[0][lid] == 1.0) and np.all(cl.vel_bc[0][~lid] == 0.0)
    assert np.all(cl.vel_bc[1] == 0.0)


def test_cavity_at_a_million_nodes():
    cl = clouds.cavity_2d(1000)
    assert cl.nv == 1_004_000 and int(cl.boundary.sum()) == 4000


def test_cube_nodes_and_faces():
    n = 10
    cl = clouds.cube_3d(n)
    ni = n ** 3
    assert cl.nv == ni + 6 * n * n and cl.dim == 3
    assert int(cl.boundary.sum()) == 6 * n * n
    b, nrm = cl.xyz[ni:], cl.normal[ni:]
    on_face = np.isclose(b, 0.0) | np.isclose(b, 1.0)
    assert np.all(on_face.sum(1) == 1)
    assert np.allclose(np.linalg.norm(nrm, axis=1), 1.0)
    assert np.all((nrm != 0) == on_face)
    assert np.all(nrm[np.isclose(b, 1.0)] == 1.0) and np.all(nrm[np.isclose(b, 0.0)] == -1.0)
    lid = cl.boundary & np.isclose(cl.xyz[:, 1], 1.0)
    assert np.all(cl.vel_bc[0][lid] == 1.0) and cl.vel_bc[0][~lid].max() == 0.0
    assert 128 ** 3 + 6 * 128 ** 2 == 2_195_456


def test_channel_with_cylinder():
    cl = clouds.channel_2d(0.05, seed=2)
    kind = cl.meta["kind"]
    x, y = cl.xyz[:, 0], cl.xyz[:, 1]
    cx, cy = cl.meta["centre"]
    r = np.hypot(x - cx, y - cy)
    inner = kind == 0
    assert np.all(r[inner] > cl.meta["radius"]) and np.all((x >= 0) & (x <= 8) & (y >= 0) & (y <= 1))
    cyl = kind == 4
    assert np.allclose(r[cyl], cl.meta["radius"])
    # normals point out of the fluid: into the cylinder on its surface
    assert np.allclose((cl.normal[cyl] * np.stack([x[cyl] - cx, y[cyl] - cy], 1)).sum(1),
                       -cl.meta["radius"])
    assert np.allclose(np.linalg.norm(cl.normal[cl.boundary], axis=1), 1.0)
    # parabolic inflow of mean 1, pressure fixed at the outlet only
    inlet = kind == 2
    assert np.isclose(np.mean(cl.vel_bc[0][inlet]), 1.0, rtol=1e-2)
    assert np.array_equal(cl.p_dirichlet, kind == 3)
    assert not (cl.u_dirichlet & (kind == 3)).any()


@pytest.mark.parametrize("make", [lambda s: clouds.cavity_2d(40, seed=s),
                                  lambda s: clouds.cube_3d(6, seed=s),
                                  lambda s: clouds.channel_2d(0.05, seed=s)])
def test_clouds_are_reproducible_from_the_seed(make):
    a, b, c = make(11), make(11), make(12)
    assert np.array_equal(a.xyz, b.xyz)
    assert a.nv == c.nv or a.name == "channel_2d"
    assert not np.array_equal(a.xyz[:10], c.xyz[:10])
