"""cudaBVH_traceClosestHostNoAlloc: the allocation-free closest-hit entry
point, for callers that cannot allocate device memory while tracing (for
instance a Vulkan layer on the application's render thread, where a
cudaMalloc can stall the frame and the application owns the memory budget).

Its results must equal cudaBVH_traceClosestHost's, call after call: checked
here in this process (after the rest of the suite when the whole suite
runs) and, by `test_no_alloc_in_a_fresh_process`, in a new Python process
whose first trace is this entry point (so its first call there looks up
the scratch array's device address).  Free device memory must not change across
calls, on the default stream or a created one, and a call rejected for size
must leave the next call clean.  The file name makes pytest collect it last,
so a stop-at-first-failure run has already run everything else.
"""
import subprocess
import sys
import textwrap
from pathlib import Path

import numpy as np
import pytest

from rtb200 import lib, scenes
from rtb200.scenes import HIT_DTYPE

pytestmark = pytest.mark.gpu

MAX_RAYS = 65536
RT_ERR_CAPACITY = -6
ROOT = Path(__file__).resolve().parents[1]


def _noalloc(bvh, rays, stream=None):
    hits = np.zeros(rays.shape[0], HIT_DTYPE)
    rc = lib.load().cudaBVH_traceClosestHostNoAlloc(bvh.h, rays.ctypes.data, rays.shape[0], hits.ctypes.data,
                                                     stream)
    return rc, hits


def _assert_same(got, ref):
    assert np.array_equal(got["prim"], ref["prim"])
    for f in ("t", "u", "v"):
        assert np.array_equal(got[f].view(np.uint32), ref[f].view(np.uint32)), f


def test_no_alloc_matches_allocating_entry_point_twice(cuda):
    import torch
    tris = scenes.scene_spheres_100k(3)[:20002]
    bvh = lib.BVH(tris)
    batches = [np.ascontiguousarray(scenes.random_rays(seed, n)) for seed, n in ((7, 40000), (8, MAX_RAYS))]
    refs = [bvh.closest_host(r) for r in batches]  # the allocating path grows its staging here
    stream = torch.cuda.Stream()
    rc, _ = _noalloc(bvh, batches[0])  # warm: the first call looks up the scratch address
    assert rc == 0, lib.last_error()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    # two different batches in a row, then again on a created stream: no call may
    # see the previous one's rays, hits, counter or status
    for s in (None, stream.cuda_stream):
        for rays, ref in zip(batches, refs):
            rc, got = _noalloc(bvh, rays, s)
            assert rc == 0, lib.last_error()
            _assert_same(got, ref)
            assert (ref["prim"] >= 0).mean() > 0.05
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0, "device memory changed across allocation-free calls"


def test_no_alloc_rejects_oversized_batches_then_traces_cleanly(cuda):
    bvh = lib.BVH(scenes.scene_spheres_100k(3)[:2002])
    rays = np.ascontiguousarray(scenes.random_rays(9, MAX_RAYS + 1))
    rc, _ = _noalloc(bvh, rays)
    assert rc == RT_ERR_CAPACITY and "65536" in lib.last_error()
    empty = np.zeros(0, scenes.RAY_DTYPE)
    assert lib.load().cudaBVH_traceClosestHostNoAlloc(bvh.h, empty.ctypes.data, 0, empty.ctypes.data, None) == 0
    # the next good call after a rejection: exact results, clean status
    ok = np.ascontiguousarray(rays[:MAX_RAYS])
    rc, got = _noalloc(bvh, ok)
    assert rc == 0, lib.last_error()
    _assert_same(got, bvh.closest_host(ok))


FRESH = textwrap.dedent("""
    import sys
    sys.path[:0] = [{root!r}, {pkg!r}]
    import numpy as np
    from rtb200 import lib, scenes
    from rtb200.scenes import HIT_DTYPE
    L = lib.load()
    bvh = lib.BVH(scenes.scene_spheres_100k(3)[:20002])
    outs = []
    for seed, n in ((7, 40000), (8, 65536)):
        rays = np.ascontiguousarray(scenes.random_rays(seed, n))
        hits = np.zeros(n, HIT_DTYPE)
        rc = L.cudaBVH_traceClosestHostNoAlloc(bvh.h, rays.ctypes.data, n, hits.ctypes.data, None)
        assert rc == 0, lib.last_error()
        ref = bvh.closest_host(rays)
        assert np.array_equal(hits.view(np.uint8), ref.view(np.uint8)), seed
        outs.append(int((ref["prim"] >= 0).sum()))
    print("fresh-process ok", outs)
""")


def test_no_alloc_in_a_fresh_process(cuda):
    code = FRESH.format(root=str(ROOT), pkg=str(ROOT / "vk-rt-cuda-raytracing_b200"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "fresh-process ok" in r.stdout
