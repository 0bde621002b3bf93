"""Parity at the benchmark's full sizes.

Config 1 (the headline workload, the same seeds and sizes bench.py times):
a 2,000,000-triangle scene of sphere and box meshes, the 1920x1080 primary
pass, then 2M cosine-weighted diffuse bounce rays with a 0.001 * normal
origin offset (multi_bounce.cu:343-356 form; closest hit) and 2M area-light
shadow rays (any hit), both made on the GPU by cudaBVH_generateRays from
the primary hits and checked bit for bit against the oracle's restatement
of the generator.  Every ray is compared with the oracle's restated
traversal (layer/shaders/bvh2_stackless.comp:37-76 with the Moller-Trumbore
arithmetic of layer/cuda_bvh_backend.cu:143-157) over the restated
reference builder's BVH: primitive ids, t, u and v bit-identical, occlusion
flags identical.

Config 2: the wavefront path tracer at its benchmark size (1920x1080, 8 spp,
<= 4 bounces, Russian roulette from bounce 2, 64 instances over 16 BLASes
with 5,000,000 triangles) against the FP64 oracle path tracer on 4,096
seeded pixels: mean relative error <= 1e-4 (the bar for radiance under
per-pixel Philox streams).
"""
import numpy as np
import pytest

from oracle import oracle as O
from rtb200 import lib, scenes
from rtb200.scenes import HIT_DTYPE

pytestmark = pytest.mark.gpu

N_TRIS = 2_000_000
N_RAYS = 2_000_000


def _trace(torch, bvh, rays, any_hit=False):
    d_rays = torch.from_numpy(np.ascontiguousarray(rays).view(np.uint8).copy()).cuda()
    n = rays.shape[0]
    out = torch.empty(n * (1 if any_hit else 16), dtype=torch.uint8, device="cuda")
    (bvh.any if any_hit else bvh.closest)(d_rays, n, out)
    torch.cuda.synchronize()
    res = out.cpu().numpy()
    return res if any_hit else res.view(HIT_DTYPE)


def _assert_bitexact(got, ref, what):
    bad = ((got["prim"] != ref["prim"]) | (got["t"].view(np.uint32) != ref["t"].view(np.uint32)) |
           (got["u"].view(np.uint32) != ref["u"].view(np.uint32)) | (got["v"].view(np.uint32) != ref["v"].view(np.uint32)))
    idx = np.nonzero(bad)[0]
    assert idx.size == 0, f"{what}: {idx.size} of {got.shape[0]} rays differ, first {idx[:5]}"


def test_config1_fullsize_every_ray(cuda):
    import torch
    tris = scenes.scene_meshes(1, N_TRIS)
    assert tris.shape[0] == N_TRIS
    bvh = lib.BVH(tris)
    ob = O.OracleBVH(tris, nbins=32, max_leaf=4)
    prim = scenes.primary_1080p()
    ph = _trace(torch, bvh, prim)
    _assert_bitexact(ph, ob.closest(prim), "primary 1080p")
    d_prim = torch.from_numpy(prim.view(np.uint8).copy()).cuda()
    d_ph = torch.from_numpy(ph.view(np.uint8).copy()).cuda()
    made = []
    for kind, seed in ((lib.RT_GEN_DIFFUSE, 3), (lib.RT_GEN_SHADOW, 4)):
        d_out = torch.empty(N_RAYS * 32, dtype=torch.uint8, device="cuda")
        d_cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
        bvh.generate_rays(d_prim, d_ph, prim.shape[0], d_out, d_cnt, kind=kind, count=N_RAYS, seed=seed)
        torch.cuda.synchronize()
        assert int(d_cnt.item()) == N_RAYS
        rays = d_out.cpu().numpy().view(scenes.RAY_DTYPE)
        ref, _ = O.generate_rays(tris, prim, ph, kind, count=N_RAYS, seed=seed)
        assert np.array_equal(rays.view(np.uint32), ref.view(np.uint32)), f"generated rays (kind {kind}) differ"
        made.append(rays)
    dif, sha = made
    got = _trace(torch, bvh, dif)
    _assert_bitexact(got, ob.closest(dif), "2M diffuse closest hit")
    assert 0.3 < (got["prim"] >= 0).mean() < 0.6
    occ = _trace(torch, bvh, sha, any_hit=True)
    ref = ob.any(sha)
    bad = np.nonzero(occ != ref)[0]
    assert bad.size == 0, f"2M shadow any hit: {bad.size} flags differ, first {bad[:5]}"
    # the host-buffer entry point the bench's end-to-end leg calls gives the same records
    host = bvh.closest_host(dif)
    assert np.array_equal(host.view(np.uint8), got.view(np.uint8))


def test_config2_pathtracer_fullres_vs_fp64_oracle(cuda):
    import torch
    blases, xf, bidx, alb, emi = scenes.instanced_scene(2, 5_000_000, nblas=16, ninst=64, world=100.0,
                                                        emissive_frac=0.05)
    assert sum(t.shape[0] for t in blases) == 5_000_000
    bvhs = [lib.BVH(t) for t in blases]
    tl = lib.TLAS(bvhs, xf, bidx)
    pt = lib.PathTracer(tl, alb, emi)
    W, H, spp = 1920, 1080, 8
    cam = lib.make_camera(scenes.PT_CAM_EYE, scenes.PT_CAM_TARGET, vfov=50.0)
    d_rgb = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    pt.render(cam, W, H, spp, 4, 2, 1, d_rgb)
    torch.cuda.synchronize()
    img = d_rgb.cpu().numpy().reshape(-1, 3).astype(np.float64)
    st = pt.stats()
    assert st["extension_rays"] > W * H * spp and st["shadow_rays"] > 0
    orc = O.OraclePT(blases, xf, bidx, tl.inverse(), alb, emi)
    rs = np.random.RandomState(0)
    px = np.sort(rs.choice(W * H, 4096, replace=False)).astype(np.int32)
    ref, _ = orc.pixels(lib.camera_basis(cam, W, H), W, H, spp, px, 4, 2, 1)
    g = img[px]
    mre = float(np.abs(g - ref).sum() / max(np.abs(ref).sum(), 1e-30))
    assert mre <= 1e-4, mre
    assert np.abs(ref).sum() > 0
    assert np.isfinite(img).all()
