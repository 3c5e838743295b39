"""Seeded synthetic point clouds (the POINTS inputs of the solver).

The reference reads gmsh meshes (points.cpp:27-73) and keeps, per node, its
coordinates, a boundary flag and an outward unit normal (class.hpp:96-140);
boundary-condition flags and values are set by the driver.  These generators
build the same data in memory for the benchmark geometries:

  cavity_2d(nx)      unit square, nx*nx jittered interior nodes at
                     ((i+1/2)h, (j+1/2)h) +/- 0.2h, 4*nx boundary nodes at
                     (i+1/2)h on the sides (corners absent, as the reference
                     deletes corner nodes, points.cpp:323-352); lid u=1 at y=1.
  cube_3d(n)         unit cube, n^3 jittered interior nodes and 6*n^2 face
                     nodes (edges and corners absent); lid u=1 on y=1.
  channel_2d(h)      [0,8]x[0,1] with a circular obstacle r=0.1 at (1,0.5):
                     parabolic inlet, no-slip walls and cylinder, p=0 outlet.

Jitter is drawn from numpy's Philox-4x32-10 generator keyed by `seed`, so every
run and every process sees the same cloud.  Interior nodes come first in
row-major grid order (good locality for the stencil gathers), boundary nodes
after them.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

DEFAULT_SEED = 20261203


@dataclass
class Cloud:
    name: str
    xyz: np.ndarray            # (nv, dim) float64
    boundary: np.ndarray       # (nv,) bool
    normal: np.ndarray         # (nv, dim) float64, zero at interior nodes
    u_dirichlet: np.ndarray    # (nv,) bool
    v_dirichlet: np.ndarray
    p_dirichlet: np.ndarray
    w_dirichlet: np.ndarray | None = None
    vel_bc: np.ndarray | None = None   # (dim, nv) initial field carrying the BC values
    h: float = 0.0
    meta: dict = field(default_factory=dict)

    @property
    def nv(self) -> int:
        return self.xyz.shape[0]

    @property
    def dim(self) -> int:
        return self.xyz.shape[1]


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(key=seed))


def cavity_2d(nx: int, jitter: float = 0.2, seed: int = DEFAULT_SEED, lid: float = 1.0) -> Cloud:
    h = 1.0 / nx
    c = (np.arange(nx) + 0.5) * h
    X, Y = np.meshgrid(c, c, indexing="xy")  # row-major: y outer, x inner
    inner = np.stack([X.ravel(), Y.ravel()], 1)
    inner += _rng(seed).uniform(-jitter * h, jitter * h, size=inner.shape)
    z, o = np.zeros(nx), np.ones(nx)
    bxy = np.concatenate([np.stack([c, z], 1), np.stack([c, o], 1),
                          np.stack([z, c], 1), np.stack([o, c], 1)])
    bn = np.concatenate([np.tile([0.0, -1.0], (nx, 1)), np.tile([0.0, 1.0], (nx, 1)),
                         np.tile([-1.0, 0.0], (nx, 1)), np.tile([1.0, 0.0], (nx, 1))])
    xyz = np.concatenate([inner, bxy])
    nv = xyz.shape[0]
    bnd = np.zeros(nv, bool)
    bnd[nx * nx:] = True
    normal = np.zeros((nv, 2))
    normal[nx * nx:] = bn
    vel = np.zeros((2, nv))
    top = nx * nx + nx + np.arange(nx)
    vel[0, top] = lid
    return Cloud("cavity_2d", xyz, bnd, normal, u_dirichlet=bnd.copy(), v_dirichlet=bnd.copy(),
                 p_dirichlet=np.zeros(nv, bool), vel_bc=vel, h=h,
                 meta={"nx": nx, "jitter": jitter, "seed": seed})


def cube_3d(n: int, jitter: float = 0.2, seed: int = DEFAULT_SEED, lid: float = 1.0) -> Cloud:
    h = 1.0 / n
    c = (np.arange(n) + 0.5) * h
    Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    inner = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    inner += _rng(seed).uniform(-jitter * h, jitter * h, size=inner.shape)
    A, B = np.meshgrid(c, c, indexing="ij")
    a, b = A.ravel(), B.ravel()
    zero, one = np.zeros_like(a), np.ones_like(a)
    faces, normals = [], []
    for axis in range(3):
        for side, val in ((0, zero), (1, one)):
            p = np.empty((a.size, 3))
            others = [q for q in range(3) if q != axis]
            p[:, axis] = val
            p[:, others[0]] = a
            p[:, others[1]] = b
            nrm = np.zeros(3)
            nrm[axis] = 1.0 if side else -1.0
            faces.append(p)
            normals.append(np.tile(nrm, (a.size, 1)))
    xyz = np.concatenate([inner] + faces)
    nv = xyz.shape[0]
    ni = n ** 3
    bnd = np.zeros(nv, bool)
    bnd[ni:] = True
    normal = np.zeros((nv, 3))
    normal[ni:] = np.concatenate(normals)
    vel = np.zeros((3, nv))
    lid_nodes = ni + 3 * a.size + np.arange(a.size)  # axis 1 (y), side 1
    vel[0, lid_nodes] = lid
    return Cloud("cube_3d", xyz, bnd, normal, u_dirichlet=bnd.copy(), v_dirichlet=bnd.copy(),
                 w_dirichlet=bnd.copy(), p_dirichlet=np.zeros(nv, bool), vel_bc=vel, h=h,
                 meta={"n": n, "jitter": jitter, "seed": seed})


def channel_2d(h: float = 2.828e-3, jitter: float = 0.2, seed: int = DEFAULT_SEED,
               length: float = 8.0, radius: float = 0.1, centre=(1.0, 0.5),
               u_mean: float = 1.0) -> Cloud:
    nx, ny = int(round(length / h)), int(round(1.0 / h))
    hx, hy = length / nx, 1.0 / ny
    cx, cy = (np.arange(nx) + 0.5) * hx, (np.arange(ny) + 0.5) * hy
    X, Y = np.meshgrid(cx, cy, indexing="xy")
    inner = np.stack([X.ravel(), Y.ravel()], 1)
    inner += _rng(seed).uniform(-jitter, jitter, size=inner.shape) * np.array([hx, hy])
    hm = 0.5 * (hx + hy)
    dc = np.sqrt(((inner - np.array(centre)) ** 2).sum(1))
    inner = inner[dc > radius + 0.5 * hm]
    nc = int(round(2 * np.pi * radius / hm))
    th = (np.arange(nc) + 0.5) * 2 * np.pi / nc
    circ = np.stack([centre[0] + radius * np.cos(th), centre[1] + radius * np.sin(th)], 1)
    circ_n = -np.stack([np.cos(th), np.sin(th)], 1)  # outward from the fluid = into the cylinder
    zx, ox = np.zeros(nx), np.ones(nx)
    zy = np.zeros(ny)
    parts = [np.stack([cx, zx], 1), np.stack([cx, ox], 1), np.stack([zy, cy], 1),
             np.stack([zy + length, cy], 1), circ]
    norms = [np.tile([0.0, -1.0], (nx, 1)), np.tile([0.0, 1.0], (nx, 1)),
             np.tile([-1.0, 0.0], (ny, 1)), np.tile([1.0, 0.0], (ny, 1)), circ_n]
    ni = inner.shape[0]
    xyz = np.concatenate([inner] + parts)
    nv = xyz.shape[0]
    bnd = np.zeros(nv, bool)
    bnd[ni:] = True
    normal = np.zeros((nv, 2))
    normal[ni:] = np.concatenate(norms)
    kind = np.zeros(nv, np.int8)  # 0 interior 1 wall 2 inlet 3 outlet 4 cylinder
    o = ni
    kind[o:o + 2 * nx] = 1
    o += 2 * nx
    kind[o:o + ny] = 2
    o += ny
    kind[o:o + ny] = 3
    o += ny
    kind[o:] = 4
    outlet = kind == 3
    vel = np.zeros((2, nv))
    inlet = kind == 2
    yy = xyz[inlet, 1]
    vel[0, inlet] = 6.0 * u_mean * yy * (1.0 - yy)
    return Cloud("channel_2d", xyz, bnd, normal, u_dirichlet=bnd & ~outlet,
                 v_dirichlet=bnd & ~outlet, p_dirichlet=outlet.copy(), vel_bc=vel, h=hm,
                 meta={"nx": nx, "ny": ny, "kind": kind, "jitter": jitter, "seed": seed,
                       "radius": radius, "centre": centre})


def from_arrays(name, xyz, boundary, normal, u_dirichlet=None, v_dirichlet=None,
                p_dirichlet=None) -> Cloud:
    """Wrap externally built coordinates (e.g. a gmsh reader's output)."""
    nv = xyz.shape[0]
    b = np.asarray(boundary, bool)
    return Cloud(name, np.ascontiguousarray(xyz, np.float64), b,
                 np.ascontiguousarray(normal, np.float64),
                 u_dirichlet=b.copy() if u_dirichlet is None else u_dirichlet,
                 v_dirichlet=b.copy() if v_dirichlet is None else v_dirichlet,
                 p_dirichlet=np.zeros(nv, bool) if p_dirichlet is None else p_dirichlet,
                 vel_bc=np.zeros((xyz.shape[1], nv)))
