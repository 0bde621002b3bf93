"""One handle traced from several host threads and streams at once.

The reference keeps its ray counters in global device symbols, so two traces
in flight at once share them and race (layer/cuda_bvh_backend.cu:41-42,
766-768).  Here every launch draws its own work counter from the handle's
ring with an atomic index, so concurrent traces on one handle must give
byte for byte the results of the same traces run one after another.  A TLAS
whose instances are replaced while other threads trace must give each trace
wholly the old or wholly the new instances' results.
"""
import threading

import numpy as np
import pytest

from rtb200 import lib, scenes

pytestmark = pytest.mark.gpu


def _run_threads(fns):
    errors = []

    def wrap(f):
        try:
            f()
        except BaseException as e:  # reported by the main thread
            errors.append(e)

    ths = [threading.Thread(target=wrap, args=(f,)) for f in fns]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    if errors:
        raise errors[0]


def test_threads_and_streams_on_one_handle(cuda):
    import torch
    tris = scenes.scene_meshes(5, 300_000)
    bvh = lib.BVH(tris)
    batches = [np.ascontiguousarray(scenes.random_rays(70 + k, 150_000 + 7919 * k, box=80.0)) for k in range(8)]
    d_rays = [torch.from_numpy(b.view(np.uint8).copy()).cuda() for b in batches]
    # serial results, default stream
    serial_c, serial_a = [], []
    for b, d in zip(batches, d_rays):
        h = torch.empty(b.shape[0] * 16, dtype=torch.uint8, device="cuda")
        o = torch.empty(b.shape[0], dtype=torch.uint8, device="cuda")
        bvh.closest(d, b.shape[0], h)
        bvh.any(d, b.shape[0], o)
        torch.cuda.synchronize()
        serial_c.append(h.cpu())
        serial_a.append(o.cpu())
    host_ref = bvh.closest_host(batches[0])
    # 4 host threads x 2 streams each, every thread tracing every batch, both hit kinds,
    # several rounds, with host-buffer calls on the same handle mixed in
    streams = [[torch.cuda.Stream() for _ in range(2)] for _ in range(4)]
    outs = {}

    def worker(t):
        for rnd in range(3):
            for k, (b, d) in enumerate(zip(batches, d_rays)):
                s = streams[t][(k + rnd) % 2]
                with torch.cuda.stream(s):
                    h = torch.empty(b.shape[0] * 16, dtype=torch.uint8, device="cuda")
                    o = torch.empty(b.shape[0], dtype=torch.uint8, device="cuda")
                bvh.closest(d, b.shape[0], h, stream=s)
                bvh.any(d, b.shape[0], o, stream=s)
                outs[(t, rnd, k)] = (h, o, s)
            if t == 0:
                got = bvh.closest_host(batches[0])
                assert np.array_equal(got.view(np.uint8), host_ref.view(np.uint8))

    _run_threads([lambda t=t: worker(t) for t in range(4)])
    torch.cuda.synchronize()
    assert len(outs) == 4 * 3 * 8
    for (t, rnd, k), (h, o, s) in outs.items():
        assert torch.equal(h.cpu(), serial_c[k]), (t, rnd, k)
        assert torch.equal(o.cpu(), serial_a[k]), (t, rnd, k)
    assert bvh.status() == 0


def test_tlas_updates_while_other_threads_trace(cuda):
    import torch
    blases = [lib.BVH(scenes.scene_meshes(40 + i, 20_000, box=30.0, lo=500, hi=3000, ground=False))
              for i in range(3)]
    n = 24

    def instances(seed):
        r = np.random.RandomState(seed)
        xf = [np.concatenate([scenes.rotations(r.uniform(size=(1, 3)))[0] * r.uniform(0.5, 2.0),
                              r.uniform(-30, 30, 3)[:, None]], 1).astype(np.float32) for _ in range(n)]
        return np.array(xf), r.randint(0, 3, n)

    xa, ba = instances(11)
    xb, bb = instances(12)
    rays = scenes.random_rays(80, 200_000, box=70.0)
    d_rays = torch.from_numpy(rays.view(np.uint8).copy()).cuda()
    want = []
    for xf, bi in ((xa, ba), (xb, bb)):
        tl = lib.TLAS(blases, xf, bi)
        h = torch.empty(rays.shape[0] * 16, dtype=torch.uint8, device="cuda")
        tl.closest(d_rays, rays.shape[0], h)
        torch.cuda.synchronize()
        want.append(h.cpu())
        tl.close()
    assert not torch.equal(want[0], want[1])
    shared = lib.TLAS(blases, xa, ba)
    stop = threading.Event()
    seen = [[0, 0] for _ in range(2)]

    def tracer(i):
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            h = torch.empty(rays.shape[0] * 16, dtype=torch.uint8, device="cuda")
        it = 0
        while it < 4 or not stop.is_set():
            it += 1
            shared.closest(d_rays, rays.shape[0], h, stream=s)
            s.synchronize()
            got = h.cpu()
            k = 0 if torch.equal(got, want[0]) else 1
            assert k == 0 or torch.equal(got, want[1]), "a trace saw a mix of old and new instances"
            seen[i][k] += 1

    def updater():
        try:
            for j in range(40):
                xf, bi = ((xb, bb), (xa, ba))[j % 2]
                shared.set_transforms(xf, bi)
        finally:
            stop.set()

    _run_threads([lambda: tracer(0), lambda: tracer(1), updater])
    assert min(map(sum, seen)) >= 4
    assert lib.load().cudaTLAS_getStatus(shared.h, None) == 0
    shared.close()
