"""Served form (rtServer_*): results are the same alone and in the mix.

Each request's results must be byte-identical to the plain per-call entry
points (cudaBVH_traceClosest / cudaBVH_traceAny on the scene's own BVH),
whether it runs alone or among many others of different sizes, scenes and
hit kinds, chunked across wavefronts and held back by admission.
"""
import threading

import numpy as np
import pytest

from rtb200 import lib, scenes
from rtb200.scenes import HIT_DTYPE

pytestmark = pytest.mark.gpu


def _pinned(torch, nbytes):
    return torch.empty(max(nbytes, 1), dtype=torch.uint8, pin_memory=True)


@pytest.fixture(scope="module")
def served(cuda):
    import torch
    sizes = [3000, 25000, 60000, 9000]
    tris = [scenes.scene_meshes(300 + i, n, box=40.0, lo=200, hi=3000, ground=(i % 2 == 0))
            for i, n in enumerate(sizes)]
    bvhs = [lib.BVH(t) for t in tris]
    rs = np.random.RandomState(11)
    reqs = []
    for k in range(48):
        scene = int(rs.randint(len(tris)))
        n = int(np.exp(rs.uniform(np.log(1), np.log(150_000))))
        any_hit = bool(rs.rand() < 0.3)
        rays = scenes.random_rays(400 + k, n, box=50.0)
        if any_hit:
            rays["tmax"] = np.float32(rs.uniform(5.0, 60.0))
        reqs.append((scene, any_hit, rays))
    reqs.append((1, False, scenes.random_rays(999, 0)))  # an empty request
    # expected results from the plain per-call path on each scene's own BVH
    expect = []
    for scene, any_hit, rays in reqs:
        n = rays.shape[0]
        if n == 0:
            expect.append(np.zeros(0, np.uint8))
            continue
        d_r = torch.from_numpy(rays.view(np.uint8).copy()).cuda()
        d_o = torch.empty(n * (1 if any_hit else 16), dtype=torch.uint8, device="cuda")
        (bvhs[scene].any if any_hit else bvhs[scene].closest)(d_r, n, d_o)
        torch.cuda.synchronize()
        expect.append(d_o.cpu().numpy())
    return tris, bvhs, reqs, expect


def _server(bvhs, **kw):
    srv = lib.Server(**kw)
    ids = [srv.add_scene(b) for b in bvhs]
    assert ids == list(range(len(bvhs)))
    return srv


def _run(torch, srv, reqs, concurrent):
    """Submits every request (one at a time, or all at once from two
    threads) with pinned host buffers; returns results and request infos."""
    hin = [_pinned(torch, r[2].nbytes) for r in reqs]
    hout = [_pinned(torch, r[2].shape[0] * (1 if r[1] else 16)) for r in reqs]
    for h, r in zip(hin, reqs):
        if r[2].nbytes:
            h.numpy()[: r[2].nbytes] = r[2].view(np.uint8)
    infos = [None] * len(reqs)

    def one(i):
        scene, any_hit, rays = reqs[i]
        return srv.submit(scene, any_hit, hin[i].data_ptr(), rays.shape[0], hout[i].data_ptr())

    if not concurrent:
        for i in range(len(reqs)):
            infos[i] = srv.wait(one(i), timeout_ms=60_000)
    else:
        tickets = [None] * len(reqs)

        def submitter(idx):
            for i in idx:
                tickets[i] = one(i)

        th = [threading.Thread(target=submitter, args=(list(range(j, len(reqs), 2)),)) for j in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for i in range(len(reqs)):
            infos[i] = srv.wait(tickets[i], timeout_ms=60_000)
    outs = [hout[i].numpy()[: reqs[i][2].shape[0] * (1 if reqs[i][1] else 16)].copy() for i in range(len(reqs))]
    return outs, infos


def test_served_alone_equals_mix_equals_plain(served):
    import torch
    tris, bvhs, reqs, expect = served
    # small wavefronts, chunks and staging pool: requests are split across
    # wavefronts and wait for admission while others are in flight
    srv = _server(bvhs, pool_bytes=24 << 20, wave_rays=60_000, chunk_rays=20_000, max_inflight=6, max_waves=3)
    alone, _ = _run(torch, srv, reqs, concurrent=False)
    mix, infos = _run(torch, srv, reqs, concurrent=True)
    for i, (a, m, e) in enumerate(zip(alone, mix, expect)):
        assert np.array_equal(a, e), f"request {i} alone differs from the plain path"
        assert np.array_equal(m, e), f"request {i} in the mix differs from the plain path"
    assert all(inf["status"] == 0 for inf in infos)
    assert max(inf["waves"] for inf in infos) > 1  # some requests were chunked over several wavefronts
    st = srv.stats()
    assert st["requests_done"] == 2 * len(reqs)
    assert st["rays_done"] == 2 * sum(r[2].shape[0] for r in reqs)
    assert st["peak_pool_used"] <= 24 << 20
    assert st["num_scenes"] == len(bvhs)
    hits = np.concatenate([m.view(HIT_DTYPE) for m, r in zip(mix, reqs) if not r[1] and r[2].shape[0]])
    assert 0.05 < (hits["prim"] >= 0).mean() < 0.95
    srv.close()


def test_served_device_buffers(served):
    import torch
    tris, bvhs, reqs, expect = served
    srv = _server(bvhs, pool_bytes=8 << 20, wave_rays=100_000, chunk_rays=30_000)
    bufs, tickets = [], []
    for scene, any_hit, rays in reqs[:16]:
        n = rays.shape[0]
        d_r = torch.from_numpy(rays.view(np.uint8).copy()).cuda() if n else torch.empty(32, dtype=torch.uint8,
                                                                                            device="cuda")
        d_o = torch.empty(max(n * (1 if any_hit else 16), 1), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        tickets.append(srv.submit(scene, any_hit, d_r.data_ptr(), n, d_o.data_ptr(), device=True))
        bufs.append((d_r, d_o))
    for i, t in enumerate(tickets):
        srv.wait(t, timeout_ms=60_000)
        n = reqs[i][2].shape[0] * (1 if reqs[i][1] else 16)
        assert np.array_equal(bufs[i][1].cpu().numpy()[:n], expect[i])
    srv.close()


def test_served_admission_limits(served):
    import torch
    tris, bvhs, reqs, expect = served
    srv = _server(bvhs[:1], pool_bytes=1 << 20)
    big = scenes.random_rays(5, 40_000)  # 40,000 * 48 bytes > 1 MiB: can never be admitted
    h = _pinned(torch, big.nbytes)
    o = _pinned(torch, 40_000 * 16)
    with pytest.raises(lib.RtError):
        srv.submit(0, False, h.data_ptr(), 40_000, o.data_ptr())
    with pytest.raises(lib.RtError):
        srv.submit(7, False, h.data_ptr(), 10, o.data_ptr())  # no such scene
    with pytest.raises(lib.RtError):
        srv.wait(123456)  # unknown ticket
    srv.close()
    # the HBM budget covers resident scenes too
    tight = lib.Server(hbm_budget_bytes=(1 << 20) + 4096, pool_bytes=1 << 20)
    with pytest.raises(lib.RtError):
        tight.add_scene(bvhs[2])
    tight.close()


def test_misaligned_device_pointers_are_rejected(served):
    """Device paths write 16-byte hit records; a misaligned pointer is an
    argument error reported before any launch, never a GPU fault."""
    import torch
    tris, bvhs, reqs, expect = served
    rays = reqs[0][2][:64]
    d_r = torch.from_numpy(rays.view(np.uint8).copy()).cuda()
    d_o = torch.empty(64 * 16 + 16, dtype=torch.uint8, device="cuda")
    with pytest.raises(lib.RtError):
        bvhs[0].closest(d_r, 64, d_o[4:])  # hits off by 4 bytes
    with pytest.raises(lib.RtError):
        bvhs[0].closest(d_r[8:], 63, d_o)  # rays off by 8 bytes
    srv = _server(bvhs[:1])
    with pytest.raises(lib.RtError):
        srv.submit(0, False, d_r.data_ptr(), 64, d_o.data_ptr() + 4, device=True)
    srv.close()
    bvhs[0].closest(d_r, 64, d_o)  # the aligned call still works
    torch.cuda.synchronize()
