"""cudaBVH_generateRays: next-bounce rays made on the device.

The reference builds its incoherent secondary rays with genAndCompact
(multi_bounce.cu:281-362: hit point, facing normal, cosine-weighted bounce,
origin offset 0.001 * n, block compaction of the live rays).  The library's
generator must equal the oracle's restatement bit for bit (rays, source
indices, count), keep the hits' input order (deterministic compaction), drop
misses and hits whose primitive is not in the BVH, and handle empty batches.
"""
import numpy as np
import pytest

from oracle import oracle as O
from rtb200 import lib, scenes
from rtb200.scenes import HIT_DTYPE, RAY_DTYPE

pytestmark = pytest.mark.gpu


def _gen(torch, bvh, rays, hits, kind, count=0, **kw):
    n = rays.shape[0]
    d_r = torch.from_numpy(np.ascontiguousarray(rays).view(np.uint8).copy()).cuda()
    d_h = torch.from_numpy(np.ascontiguousarray(hits).view(np.uint8).copy()).cuda()
    cap = max(count if count > 0 else n, 1)
    d_out = torch.full((cap * 32,), 0xAB, dtype=torch.uint8, device="cuda")
    d_src = torch.full((cap,), -7, dtype=torch.int32, device="cuda")
    d_cnt = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    bvh.generate_rays(d_r, d_h, n, d_out, d_cnt, kind=kind, count=count, d_src=d_src, **kw)
    torch.cuda.synchronize()
    m = int(d_cnt.item())
    return d_out.cpu().numpy().view(RAY_DTYPE)[:m], d_src.cpu().numpy()[:m], m


def _assert_rays_equal(a, b, what):
    assert a.shape == b.shape, (what, a.shape, b.shape)
    bad = np.nonzero(np.any(a.view(np.uint32).reshape(-1, 8) != b.view(np.uint32).reshape(-1, 8), axis=1))[0]
    assert bad.size == 0, f"{what}: {bad.size} rays differ, first {bad[:5]}: {a[bad[:2]]} vs {b[bad[:2]]}"


def test_generated_rays_equal_the_oracle(cuda):
    import torch
    tris = scenes.scene_spheres_100k(0)
    bvh = lib.BVH(tris)
    prim = scenes.primary_1080p()
    d_prim = torch.from_numpy(prim.view(np.uint8).copy()).cuda()
    d_ph = torch.empty(prim.shape[0] * 16, dtype=torch.uint8, device="cuda")
    bvh.closest(d_prim, prim.shape[0], d_ph)
    torch.cuda.synchronize()
    ph = d_ph.cpu().numpy().view(HIT_DTYPE)
    nhit = int((ph["prim"] >= 0).sum())
    assert 0.2 * prim.shape[0] < nhit < prim.shape[0]
    cases = [("diffuse, one per hit", dict(kind=lib.RT_GEN_DIFFUSE, count=0, seed=3)),
             ("diffuse, 2M cycling", dict(kind=lib.RT_GEN_DIFFUSE, count=2_000_000, seed=3)),
             ("shadow, one per hit", dict(kind=lib.RT_GEN_SHADOW, count=0, seed=4)),
             ("shadow, 2M cycling", dict(kind=lib.RT_GEN_SHADOW, count=2_000_000, seed=4, light_size=2.0))]
    for what, kw in cases:
        got, src, m = _gen(torch, bvh, prim, ph, **kw)
        ref, rsrc = O.generate_rays(tris, prim, ph, kw["kind"], count=kw["count"], seed=kw["seed"],
                                    light_size=kw.get("light_size", 1.0))
        assert m == (kw["count"] or nhit), what
        _assert_rays_equal(got, ref, what)
        assert np.array_equal(src, rsrc), what
        # compaction keeps the hits' input order
        surv = np.nonzero(ph["prim"] >= 0)[0]
        assert np.array_equal(src[:nhit], surv[: min(nhit, m)]), what
    # diffuse directions are unit vectors in the hemisphere of the facing normal
    got, src, m = _gen(torch, bvh, prim, ph, kind=lib.RT_GEN_DIFFUSE, count=0)
    p, n = scenes.hit_frame(tris, prim, ph)
    c = np.einsum("ij,ij->i", got["dir"].astype(np.float64), n.astype(np.float64))
    assert c.min() >= 0.0 and abs(c.mean() - 2.0 / 3.0) < 0.01
    assert np.allclose(np.linalg.norm(got["dir"], axis=1), 1.0, atol=1e-6)


def test_generator_edges(cuda):
    import torch
    tris = scenes.scene_spheres_100k(1)[:5002]
    bvh = lib.BVH(tris)
    rays = scenes.random_rays(31, 10_000)
    hits = bvh.closest_host(rays)
    # hits naming a primitive outside this BVH are skipped, never followed
    bogus = hits.copy()
    k = np.nonzero(bogus["prim"] >= 0)[0][:50]
    bogus["prim"][k] = tris.shape[0] + 1000
    got, src, m = _gen(torch, bvh, rays, bogus, kind=lib.RT_GEN_DIFFUSE)
    assert m == int((hits["prim"] >= 0).sum()) - k.size
    assert not np.isin(k, src).any()
    ref, rsrc = O.generate_rays(tris, rays, bogus, 0)
    _assert_rays_equal(got, ref, "bogus ids")
    # all misses: nothing, also when a count is asked for
    miss = hits.copy()
    miss["prim"] = -1
    for count in (0, 1000):
        got, src, m = _gen(torch, bvh, rays, miss, kind=lib.RT_GEN_SHADOW, count=count)
        assert m == 0
    # an empty batch
    got, src, m = _gen(torch, bvh, rays[:0], hits[:0], kind=lib.RT_GEN_DIFFUSE)
    assert m == 0
    # the rays traced back hit nothing behind their own surface: a diffuse
    # bounce leaves the surface it starts on (offset eps along the normal)
    got, src, m = _gen(torch, bvh, rays, hits, kind=lib.RT_GEN_DIFFUSE)
    back = bvh.closest_host(got)
    assert not np.any(back["prim"] == hits["prim"][src])


def test_regroup_sorts_stably_and_keeps_every_ray(cuda):
    """rtRays_regroup: a permutation of the input, ordered by the key
    (direction octant, then the origin's Morton code in the box), equal keys
    in input order; tracing the regrouped rays gives the same hits, moved."""
    import torch
    tris = scenes.scene_spheres_100k(2)[:30002]
    bvh = lib.BVH(tris)
    rays = scenes.random_rays(41, 300_001, box=120.0)
    box = np.array([-60, -60, -60, 60, 60, 60], np.float32)
    n = rays.shape[0]
    d_in = torch.from_numpy(rays.view(np.uint8).copy()).cuda()
    for kind in (lib.RT_REGROUP_MORTON, lib.RT_REGROUP_OCTANT_MORTON):
        for bits in (16, 32):
            d_out = torch.empty_like(d_in)
            d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
            lib.regroup_rays(d_in, n, box, d_out, kind=kind, key_bits=bits, d_perm=d_perm)
            torch.cuda.synchronize()
            perm = d_perm.cpu().numpy()
            out = d_out.cpu().numpy().view(RAY_DTYPE)
            assert np.array_equal(np.sort(perm), np.arange(n))
            assert np.array_equal(out.view(np.uint8), rays[perm].view(np.uint8))
            # keys recomputed on the host: non-decreasing, ties in input order
            o = rays["org"].astype(np.float32)
            q = np.clip(((o - box[:3]) * (np.float32(1) / (box[3:] - box[:3])) * np.float32(1024)),
                        0, 1023).astype(np.uint64)

            def spread(v):
                v = (v | (v << np.uint64(16))) & np.uint64(0x030000FF)
                v = (v | (v << np.uint64(8))) & np.uint64(0x0300F00F)
                v = (v | (v << np.uint64(4))) & np.uint64(0x030C30C3)
                return (v | (v << np.uint64(2))) & np.uint64(0x09249249)

            m = (spread(q[:, 0]) << np.uint64(2)) | (spread(q[:, 1]) << np.uint64(1)) | spread(q[:, 2])
            if kind == lib.RT_REGROUP_OCTANT_MORTON:
                d = rays["dir"]
                octv = np.signbit(d[:, 0]).astype(np.uint64) * 4 + np.signbit(d[:, 1]).astype(np.uint64) * 2 + \
                       np.signbit(d[:, 2]).astype(np.uint64)
                key = (octv << np.uint64(29)) | (m >> np.uint64(1))
            else:
                key = m << np.uint64(2)
            if bits == 16:
                key >>= np.uint64(16)
            ks = key[perm]
            assert np.all(ks[1:] >= ks[:-1])
            ties = ks[1:] == ks[:-1]
            assert np.all(perm[1:][ties] > perm[:-1][ties])
    # the traversal result of each ray does not depend on the order
    d_out = torch.empty_like(d_in)
    d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
    lib.regroup_rays(d_in, n, box, d_out, d_perm=d_perm)
    h0 = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
    h1 = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
    bvh.closest(d_in, n, h0)
    bvh.closest(d_out, n, h1)
    torch.cuda.synchronize()
    perm = d_perm.cpu().numpy()
    a = h0.cpu().numpy().view(HIT_DTYPE)[perm]
    b = h1.cpu().numpy().view(HIT_DTYPE)
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_path_tracer_image_does_not_depend_on_regrouping_or_queue_capacity(cuda):
    """Paths are independent and each keeps its own radiance slot, so the
    image and the ray counts are bit-identical whether bounce rays are
    regrouped or not and whatever the wavefront queue capacity (the frame in
    one slice, or in slices of any size, uneven last slice included)."""
    import torch
    blases, xf, bidx, alb, emi = scenes.instanced_scene(2, 200_000, nblas=4, ninst=16, world=40.0,
                                                        emissive_frac=0.25)
    bvhs = [lib.BVH(t) for t in blases]
    tl = lib.TLAS(bvhs, xf, bidx)
    cam = lib.make_camera((0.0, 10.0, -70.0), (0.0, 0.0, 0.0), vfov=50.0)
    W, H, spp = 320, 180, 4
    imgs = []
    for bits, cap in ((0, 0), (16, 0), (32, 0), (0, 77_777), (32, 50_000), (0, 4_099)):
        pt = lib.PathTracer(tl, alb, emi)
        pt.set_regroup(bits)
        pt.set_queue_capacity(cap)
        d_rgb = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
        pt.render(cam, W, H, spp, 4, 2, 1, d_rgb)
        torch.cuda.synchronize()
        imgs.append((d_rgb.cpu().numpy(), pt.stats()))
        pt.close()
    for img, st in imgs[1:]:
        assert np.array_equal(img.view(np.uint32), imgs[0][0].view(np.uint32))
        assert st["extension_rays"] == imgs[0][1]["extension_rays"]
        assert st["shadow_rays"] == imgs[0][1]["shadow_rays"]
    assert imgs[0][0].sum() > 0


def test_path_tracer_autotune_keeps_the_image(cuda):
    import torch
    blases, xf, bidx, alb, emi = scenes.instanced_scene(3, 400_000, nblas=4, ninst=16, world=40.0,
                                                        emissive_frac=0.25)
    bvhs = [lib.BVH(t) for t in blases]
    tl = lib.TLAS(bvhs, xf, bidx)
    cam = lib.make_camera((0.0, 10.0, -70.0), (0.0, 0.0, 0.0), vfov=50.0)
    W, H, spp = 640, 360, 8
    pt = lib.PathTracer(tl, alb, emi)
    a = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    b = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    pt.render(cam, W, H, spp, 4, 2, 1, a)
    cap = pt.autotune(cam, W, H, spp, 4, 2, 1, d_rgb=b)
    assert cap == 0 or (cap % spp == 0 and cap < W * H * spp)
    b.zero_()
    pt.render(cam, W, H, spp, 4, 2, 1, b)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
