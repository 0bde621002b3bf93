"""cudaBVH_traceClosestHostNoAlloc: the allocation-free closest-hit entry
point, for callers that cannot allocate device memory while tracing (for
instance a Vulkan layer on the application's render thread).  Its results
must equal cudaBVH_traceClosestHost's, call after call, whether this file
runs alone in a fresh process or after the rest of the suite.  Collected
last on purpose (file name) so a stop-at-first-failure run has already run
everything else.
"""
import ctypes as C

import numpy as np
import pytest

from rtb200 import lib, scenes
from rtb200.scenes import HIT_DTYPE

pytestmark = pytest.mark.gpu

MAX_RAYS = 65536


def _noalloc(bvh, rays):
    hits = np.zeros(rays.shape[0], HIT_DTYPE)
    rc = lib.load().cudaBVH_traceClosestHostNoAlloc(bvh.h, rays.ctypes.data, rays.shape[0], hits.ctypes.data, None)
    return rc, hits


def test_no_alloc_matches_allocating_entry_point_twice(cuda):
    tris = scenes.scene_spheres_100k(3)[:20002]
    bvh = lib.BVH(tris)
    # two different batches in a row: the second must not see the first's state
    for seed, n in ((7, 40000), (8, MAX_RAYS)):
        rays = np.ascontiguousarray(scenes.random_rays(seed, n))
        ref = bvh.closest_host(rays)
        rc, got = _noalloc(bvh, rays)
        assert rc == 0, lib.last_error()
        assert np.array_equal(got["prim"], ref["prim"])
        assert np.array_equal(got["t"].view(np.uint32), ref["t"].view(np.uint32))
        assert np.array_equal(got["u"].view(np.uint32), ref["u"].view(np.uint32))
        assert np.array_equal(got["v"].view(np.uint32), ref["v"].view(np.uint32))
        assert (ref["prim"] >= 0).mean() > 0.05


def test_no_alloc_rejects_oversized_batches(cuda):
    bvh = lib.BVH(scenes.scene_spheres_100k(3)[:2002])
    rays = np.ascontiguousarray(scenes.random_rays(9, MAX_RAYS + 1))
    rc, _ = _noalloc(bvh, rays)
    assert rc == -6 and "65536" in lib.last_error()
    empty = np.zeros(0, scenes.RAY_DTYPE)
    assert lib.load().cudaBVH_traceClosestHostNoAlloc(bvh.h, empty.ctypes.data, 0, empty.ctypes.data, None) == 0
