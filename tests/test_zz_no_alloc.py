"""GPU: the no-allocation kNN entry point against the allocating one.

mp_knn_stencils_noalloc carves its work arrays from a fixed per-device scratch
array; its stencils must equal mp_knn_stencils' exactly (integer output), call
after call, and clouds beyond the scratch must be refused with MP_BAD_ARG.
"""
import ctypes as C

import numpy as np
import pytest

from memphys_b200 import capi, clouds

pytestmark = pytest.mark.gpu


def knn_alloc(cl, n):
    nb = np.zeros((cl.nv, n), np.int32)
    capi.check(capi.lib().mp_knn_stencils(capi.ptr(cl.xyz), capi.ptr(cl.boundary), cl.nv, cl.dim,
                                          n, capi.ptr(nb), None), "mp_knn_stencils")
    return nb


def knn_noalloc(dx, db, dn, cl, n):
    return capi.lib().mp_knn_stencils_noalloc(capi.ptr(dx), capi.ptr(db), cl.nv, cl.dim, n,
                                              capi.ptr(dn), None)


@pytest.mark.parametrize("make,n", [(lambda: clouds.cavity_2d(96, seed=11), 20),
                                    (lambda: clouds.cube_3d(14, seed=12), 30)])
def test_noalloc_matches_allocating_entry_point(mp_lib, make, n):
    cl = make()
    ref = knn_alloc(cl, n)
    dx = capi.DeviceArray.from_host(np.ascontiguousarray(cl.xyz, np.float64))
    db = capi.DeviceArray.from_host(np.ascontiguousarray(cl.boundary, np.uint8))
    for _ in range(2):  # two calls in a row reuse the same scratch
        dn = capi.DeviceArray((cl.nv, n), np.int32)
        capi.check(knn_noalloc(dx, db, dn, cl, n), "mp_knn_stencils_noalloc")
        assert np.array_equal(dn.to_host(), ref)


def test_noalloc_refuses_oversized_cloud_and_host_pointers(mp_lib):
    nv = 300_000  # the per-node arrays alone exceed the 4 MiB scratch
    dx = capi.DeviceArray((nv, 2), np.float64)
    db = capi.DeviceArray((nv,), np.uint8)
    dn = capi.DeviceArray((nv, 20), np.int32)
    L = capi.lib()
    rc = L.mp_knn_stencils_noalloc(capi.ptr(dx), capi.ptr(db), nv, 2, 20, capi.ptr(dn), None)
    assert rc == capi.MP_BAD_ARG
    msg = C.create_string_buffer(512)
    L.mp_last_error(msg, 512)
    assert b"scratch" in msg.value
    cl = clouds.cavity_2d(24, seed=1)
    nb = np.zeros((cl.nv, 12), np.int32)
    rc = L.mp_knn_stencils_noalloc(capi.ptr(cl.xyz), capi.ptr(cl.boundary), cl.nv, 2, 12,
                                   capi.ptr(nb), None)
    assert rc == capi.MP_BAD_ARG
    # a valid call still works after the refusals
    dx = capi.DeviceArray.from_host(np.ascontiguousarray(cl.xyz, np.float64))
    db = capi.DeviceArray.from_host(np.ascontiguousarray(cl.boundary, np.uint8))
    dn = capi.DeviceArray((cl.nv, 12), np.int32)
    capi.check(knn_noalloc(dx, db, dn, cl, 12), "mp_knn_stencils_noalloc")
    assert np.array_equal(dn.to_host(), knn_alloc(cl, 12))


def test_noalloc_runs_with_the_device_memory_held(mp_lib):
    """With all but a sliver of the device's free memory held by another allocation,
    the no-allocation entry point still runs (a hidden cudaMalloc would fail there) and
    leaves the free memory as it found it."""
    import torch
    cl = clouds.cavity_2d(96, seed=11)
    ref = knn_alloc(cl, 20)
    dx = capi.DeviceArray.from_host(np.ascontiguousarray(cl.xyz, np.float64))
    db = capi.DeviceArray.from_host(np.ascontiguousarray(cl.boundary, np.uint8))
    dn = capi.DeviceArray((cl.nv, 20), np.int32)
    capi.check(knn_noalloc(dx, db, dn, cl, 20), "mp_knn_stencils_noalloc")  # kernels loaded
    free0, _ = torch.cuda.mem_get_info()
    hog = capi.DeviceArray((free0 - (48 << 20),), np.uint8)  # leave 48 MiB
    try:
        free1, _ = torch.cuda.mem_get_info()
        assert free1 < (64 << 20)
        for _ in range(2):
            dn.zero()
            capi.check(knn_noalloc(dx, db, dn, cl, 20), "mp_knn_stencils_noalloc")
            assert np.array_equal(dn.to_host(), ref)
        assert torch.cuda.mem_get_info()[0] == free1
    finally:
        hog.free()
