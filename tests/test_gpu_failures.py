"""Failure paths, made on the host or by construction, never by a GPU fault.

* Stack overflow: the release traversal stack (64 entries) holds every tree
  the builder makes, so its overflow path is unreachable there.  A test build
  of the same sources with a 4-entry stack (lib/libcudabvh_b200_stack4.so,
  `make -C vk-rt-cuda-raytracing_b200/csrc teststack`) reaches it on an
  ordinary scene: the overflow must be reported (RT_ERR_STACK from the
  host-buffer call, from cudaBVH_getStatus after device-pointer calls), the
  overflowed rays reported as misses, every other ray exact, and the next
  call clean.  The reference drops stack entries silently instead
  (layer/cuda_bvh_backend.cu:179).
* Allocation failure: the host-side hook rtDebug_failAllocations makes the
  library's next device allocation fail; the call must fail cleanly with
  RT_ERR_NOMEM / NULL and a message, and the library must work afterwards.
* Bounded waits: rtServer_wait with a limit returns RT_ERR_TIMEOUT while the
  request is queued behind others, and the ticket stays valid.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import oracle as O
from rtb200 import lib, scenes
from rtb200.scenes import HIT_DTYPE

pytestmark = pytest.mark.gpu

RT_ERR_NOMEM, RT_ERR_STACK, RT_ERR_TIMEOUT = -3, -4, -5


def _stack4():
    path = lib.PKG_ROOT / "lib" / "libcudabvh_b200_stack4.so"
    if not path.exists():
        pytest.fail(f"{path} not built (make -C vk-rt-cuda-raytracing_b200/csrc teststack)")
    return lib.load(path)


def test_stack_overflow_is_reported_never_silent(cuda, monkeypatch):
    import torch
    S = _stack4()
    tris = scenes.scene_meshes(1, 400_000)
    rays = np.ascontiguousarray(scenes.random_rays(21, 60_000, box=60.0))
    ref = lib.BVH(tris).closest_host(rays)  # release library, 64-entry stack
    # validation rejects trees deeper than the stack; this build is made to overflow
    monkeypatch.setenv("RTB200_VALIDATE", "0")
    h = S.cudaBVH_build(tris.ctypes.data, tris.shape[0])
    assert h, S.rtGetLastError().decode()
    try:
        hits = np.zeros(rays.shape[0], HIT_DTYPE)
        rc = S.cudaBVH_traceClosestHost(h, rays.ctypes.data, rays.shape[0], hits.ctypes.data)
        assert rc == RT_ERR_STACK, rc
        assert "overflow" in S.rtGetLastError().decode()
        # overflowed rays are misses; every other ray is exact
        lost = (hits["prim"] < 0) & (ref["prim"] >= 0)
        assert 0 < lost.sum() < (ref["prim"] >= 0).sum()
        ok = ~lost
        assert np.array_equal(hits["prim"][ok], ref["prim"][ok])
        assert np.array_equal(hits["t"][ok].view(np.uint32), ref["t"][ok].view(np.uint32))
        # device-pointer calls queue and return; the status word records the overflow
        d_rays = torch.from_numpy(rays.view(np.uint8).copy()).cuda()
        d_hits = torch.empty(rays.shape[0] * 16, dtype=torch.uint8, device="cuda")
        st = torch.cuda.Stream()
        assert S.cudaBVH_traceClosest(h, d_rays.data_ptr(), rays.shape[0], d_hits.data_ptr(), st.cuda_stream) == 0
        assert S.cudaBVH_getStatus(h, st.cuda_stream) == RT_ERR_STACK
        assert S.cudaBVH_getStatus(h, st.cuda_stream) == 0  # read and cleared
        dev = d_hits.cpu().numpy().view(HIT_DTYPE)
        assert np.array_equal(dev["prim"], hits["prim"])
    finally:
        S.cudaBVH_destroy(h)
    # a shallow tree never overflows the small stack: RT_OK and brute-force hits
    small = scenes.scene_spheres_100k(4)[:40]
    h = S.cudaBVH_build(small.ctypes.data, small.shape[0])
    assert h
    try:
        r = np.ascontiguousarray(scenes.random_rays(22, 5000, box=8.0))
        got = np.zeros(r.shape[0], HIT_DTYPE)
        assert S.cudaBVH_traceClosestHost(h, r.ctypes.data, r.shape[0], got.ctypes.data) == 0
        want = O.brute_closest(small, r)
        assert np.array_equal(got["prim"], want["prim"])
    finally:
        S.cudaBVH_destroy(h)


def test_injected_allocation_failures_fail_cleanly(cuda):
    L = lib.load()
    tris = scenes.scene_spheres_100k(5)[:30002]
    rays = np.ascontiguousarray(scenes.random_rays(23, 50_000))
    try:
        L.rtDebug_failAllocations(0)
        with pytest.raises(lib.RtError, match="injected"):
            lib.BVH(tris)
        L.rtDebug_failAllocations(-1)
        bvh = lib.BVH(tris)
        # the host-buffer call must grow its staging for this batch: make that fail
        L.rtDebug_failAllocations(0)
        hits = np.zeros(rays.shape[0], HIT_DTYPE)
        rc = L.cudaBVH_traceClosestHost(bvh.h, rays.ctypes.data, rays.shape[0], hits.ctypes.data)
        assert rc == RT_ERR_NOMEM and "injected" in lib.last_error()
        # one allocation allowed, the next refused: a build that fails half-way
        L.rtDebug_failAllocations(1)
        with pytest.raises(lib.RtError):
            lib.BVH(tris)
    finally:
        L.rtDebug_failAllocations(-1)
    # the library works afterwards, with the handle that saw the failure
    got = bvh.closest_host(rays)
    want = O.brute_closest(tris, rays)
    assert np.array_equal(got["prim"], want["prim"])
    assert np.array_equal(got["t"].view(np.uint32), want["t"].view(np.uint32))


def test_every_build_allocation_failure_is_clean(cuda):
    """A build whose k-th device allocation fails, for every k up to the
    first that no build reaches: the one-graph build (single scene and
    batched) and the host-driven loop return the error, leave no stream
    capturing, and the next build is byte-identical to one that never
    failed."""
    L = lib.load()
    tris = scenes.scene_meshes(21, 40_000, box=30.0, lo=500, hi=4000)
    parts = [tris[:15_000], tris[15_000:15_003], tris[15_003:]]
    rays = np.ascontiguousarray(scenes.random_rays(24, 20_000, box=40.0))
    ref = lib.BVH(tris)
    want = ref.closest_host(rays)
    ref.close()

    def sweep(make):
        failed = 0
        for k in range(200):
            L.rtDebug_failAllocations(k)
            try:
                obj = make()
            except lib.RtError as e:
                assert "injected" in str(e) or "injected" in lib.last_error()
                failed += 1
                continue
            finally:
                L.rtDebug_failAllocations(-1)
            obj.close()
            return failed
        raise AssertionError("every build failed")

    try:
        assert sweep(lambda: lib.BVH(tris)) >= 3
        assert sweep(lambda: lib.Batch(parts)) >= 3
        assert sweep(lambda: lib.Batch(parts, host_loop=True)) >= 3
    finally:
        L.rtDebug_failAllocations(-1)
    bvh = lib.BVH(tris)
    try:
        got = bvh.closest_host(rays)
        assert np.array_equal(got.view(np.uint8), want.view(np.uint8))
    finally:
        bvh.close()


def test_server_wait_times_out_then_completes(cuda):
    import torch
    bvh = lib.BVH(scenes.scene_meshes(7, 300_000))
    srv = lib.Server()
    assert srv.add_scene(bvh) == 0
    n, nreq = 4 << 20, 12
    rays = scenes.random_rays(24, n, box=60.0)
    d_rays = torch.from_numpy(rays.view(np.uint8)).cuda()
    outs = [torch.empty(n * 16, dtype=torch.uint8, device="cuda") for _ in range(nreq)]
    L = lib.load()
    tickets = [srv.submit(0, False, d_rays.data_ptr(), n, o.data_ptr(), device=True) for o in outs]
    # the last request is queued behind 11 others of 4M rays each: not done within 1 ms
    info = lib.RtRequestInfo()
    rc = L.rtServer_wait(srv.h, C.c_uint64(tickets[-1]), 1, C.byref(info))
    assert rc == RT_ERR_TIMEOUT, rc
    assert "not done within" in lib.last_error()
    # the ticket stays valid: unbounded waits return every request, results correct
    for t in tickets:
        assert srv.wait(t)["status"] == 0
    ref = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
    bvh.closest(d_rays, n, ref)
    torch.cuda.synchronize()
    for o in outs:
        assert torch.equal(o, ref)
    srv.close()
