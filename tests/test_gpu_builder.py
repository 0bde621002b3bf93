"""GPU builder tiers: sizes on each side of the warp-subtree (32) and
small-task (1024) boundaries, degenerate centroid sets, and many tiny scenes
in one batched build.  Every tree passes the structural check and gives the
brute-force oracle's hits bit for bit (the hit set is defined by the
triangle test alone, so any valid tree must agree)."""
import numpy as np
import pytest

from oracle import oracle as O
from rtb200 import lib, scenes
from rtb200.scenes import HIT_DTYPE

pytestmark = pytest.mark.gpu


def _dev(torch, arr):
    return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).copy()).cuda()


def _check(tris, rays, what):
    bvh = lib.BVH(tris)
    bvh.validate()
    got = bvh.closest_host(rays)
    ref = O.brute_closest(tris, rays)
    bad = np.nonzero((got["prim"] != ref["prim"]) | (got["t"].view(np.uint32) != ref["t"].view(np.uint32)))[0]
    assert bad.size == 0, f"{what}: {bad.size} rays differ"
    return bvh


@pytest.mark.parametrize("n", [2, 3, 31, 32, 33, 64, 1023, 1024, 1025, 2049, 40000])
def test_sizes_around_the_tier_boundaries(cuda, n):
    if n >= 100:
        tris = scenes.scene_meshes(300 + n, n, box=20.0, lo=100, hi=max(min(n, 4000), 100), ground=False)
    else:  # scattered small triangles
        rs = np.random.RandomState(n)
        c = rs.uniform(-5, 5, (n, 1, 3))
        tris = (c + rs.uniform(-0.6, 0.6, (n, 3, 3))).reshape(n, 9).astype(np.float32)
    assert tris.shape[0] == n
    rays = scenes.random_rays(400 + n, 6000, box=25.0)
    _check(tris, rays, f"n={n}")


def test_degenerate_centroids(cuda):
    rs = np.random.RandomState(7)
    one = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0], np.float32)
    rays = scenes.random_rays(8, 4000, box=3.0)
    # identical triangles: every sort key ties, every binned split is empty
    for n in (5, 40, 2000):
        _check(np.repeat(one[None], n, axis=0), rays, f"{n} identical")
    # centroids on a line (two axes constant), and all in one point with different shapes
    line = np.repeat(one[None], 3000, axis=0)
    line[:, 0::3] += np.linspace(-2, 2, 3000, dtype=np.float32)[:, None]
    _check(line, rays, "line")
    pt = (rs.uniform(-1, 1, (1500, 3, 3))).astype(np.float32)
    pt -= pt.mean(axis=1, keepdims=True)  # every centroid at the origin
    _check(pt.reshape(-1, 9), rays, "one centroid")


def test_warp_subtrees_off_gives_the_same_hits(cuda, monkeypatch):
    tris = scenes.scene_meshes(31, 30000, box=20.0, lo=200, hi=3000, ground=False)
    rays = scenes.random_rays(32, 20000, box=25.0)
    a = _check(tris, rays, "warp subtrees")
    monkeypatch.setenv("RTB200_WARP_TASK", "0")
    b = _check(tris, rays, "CTA only")
    assert a.stats()["num_nodes"] > 0 and b.stats()["num_nodes"] > 0


def test_many_tiny_scenes_in_one_batch(cuda):
    import torch
    rs = np.random.RandomState(3)
    sizes = [int(s) for s in rs.randint(1, 41, 300)]
    tris = []
    for i, n in enumerate(sizes):
        c = rs.uniform(-3, 3, (n, 1, 3))
        tris.append((c + rs.uniform(-0.5, 0.5, (n, 3, 3))).reshape(n, 9).astype(np.float32))
    nr = [64] * len(sizes)
    rays = [scenes.random_rays(500 + i, k, box=4.0) for i, k in enumerate(nr)]
    off = np.concatenate([[0], np.cumsum(nr)]).astype(np.int32)
    allr = np.concatenate(rays)
    b = lib.Batch(tris)
    d_rays, d_off = _dev(torch, allr), torch.from_numpy(off).cuda()
    d_h = torch.empty(allr.shape[0] * 16, dtype=torch.uint8, device="cuda")
    b.closest(d_rays, d_off, allr.shape[0], d_h)
    torch.cuda.synchronize()
    got = d_h.cpu().numpy().view(HIT_DTYPE)
    for i, t in enumerate(tris):
        ref = O.brute_closest(t, rays[i])
        seg = got[off[i]:off[i + 1]]
        assert np.array_equal(seg["prim"], ref["prim"]), f"scene {i} ({sizes[i]} triangles)"
        assert np.array_equal(seg["t"].view(np.uint32), ref["t"].view(np.uint32)), f"scene {i}"
    b.close()
