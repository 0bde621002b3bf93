"""The oracle's restatement of the engine's 8-wide walk (no GPU needed).

* On a two-level 8-wide tree built here by hand in the library's node
  layout (child boxes quantised outward on the grid p + q * 2^e, as the
  collapse does), the walk finds exactly the brute-force Moller-Trumbore
  hits and occlusion flags.
* On the committed fixture tests/golden/bvh8_walk_2k.npz (the library's own
  nodes and triangle records for a 2,000-triangle scene, written on a B200
  by make_bvh8_walk.py), the walk reproduces the kernel's closest hits,
  occlusion flags and per-ray node-visit / triangle-test counts exactly:
  the counts bench.py turns into algorithmic bytes per ray.
"""
import math
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from rtb200 import scenes
from rtb200.scenes import RAY_DTYPE

GOLD = Path(__file__).resolve().parent / "golden"


def _grid(node_lo, node_hi, kids_lo, kids_hi):
    """Exponent byte per axis and the 8-bit child planes, rounded outward."""
    eb = [0, 0, 0]
    ql = np.zeros((3, 8), np.uint32)
    qh = np.zeros((3, 8), np.uint32)
    for a in range(3):
        ext = float(node_hi[a]) - float(node_lo[a])
        if not ext > 0.0:
            continue
        m, k = math.frexp(ext / 255.0)
        e = k - 1 if m == 0.5 else k
        if math.ldexp(255.0, e) < ext:
            e += 1
        e = min(max(e, -126), 127)
        eb[a] = e + 127
        sc = math.ldexp(1.0, e)
        for s in range(len(kids_lo)):
            ql[a, s] = min(max(math.floor((float(kids_lo[s][a]) - float(node_lo[a])) / sc), 0), 255)
            qh[a, s] = min(max(math.ceil((float(kids_hi[s][a]) - float(node_lo[a])) / sc), 0), 255)
    return eb, ql, qh


def _pack4(v):
    return int(v[0]) | int(v[1]) << 8 | int(v[2]) << 16 | int(v[3]) << 24


def _node(kids, child_base, tri_base):
    """kids: (lo, hi, meta) per slot, meta 0xFF for an inner child."""
    lo = np.min([k[0] for k in kids], axis=0).astype(np.float32)
    hi = np.max([k[1] for k in kids], axis=0).astype(np.float32)
    eb, ql, qh = _grid(lo, hi, [k[0] for k in kids], [k[1] for k in kids])
    meta = [k[2] for k in kids] + [0] * (8 - len(kids))
    imask = sum(1 << s for s, m in enumerate(meta) if m == 0xFF)
    w = np.zeros(20, np.uint32)
    w[0:3] = lo.view(np.uint32)
    w[3] = eb[0] | eb[1] << 8 | eb[2] << 16 | imask << 24
    w[4], w[5] = child_base, tri_base
    w[6], w[7] = _pack4(meta[0:4]), _pack4(meta[4:8])
    for a in range(3):
        w[8 + 4 * a: 12 + 4 * a] = [_pack4(ql[a, 0:4]), _pack4(ql[a, 4:8]), _pack4(qh[a, 0:4]), _pack4(qh[a, 4:8])]
    return w, lo, hi


def hand_built_tree(tris):
    """Root -> up to 8 inner nodes -> up to 8 leaves of <= 3 triangles each
    (triangles ordered by centroid x).  Returns (nodes (N, 20) u32, records
    (M, 12) f32)."""
    v = tris.reshape(-1, 3, 3)
    order = np.argsort(v.mean(1)[:, 0], kind="stable")
    assert len(order) <= 8 * 8 * 3
    groups = np.array_split(order, min(8, math.ceil(len(order) / 24)))
    recs, inner, kids_root = [], [], []
    for gi, g in enumerate(groups):
        leaves = np.array_split(g, math.ceil(len(g) / 3))
        kids, base = [], len(recs)
        for leaf in leaves:
            off = len(recs) - base
            for p in leaf:
                e1, e2 = v[p, 1] - v[p, 0], v[p, 2] - v[p, 0]
                recs.append(np.concatenate([v[p, 0], np.int32(p).view(np.float32).reshape(1), e1, [0], e2, [0]]))
            kids.append((v[leaf].reshape(-1, 3).min(0), v[leaf].reshape(-1, 3).max(0), len(leaf) << 5 | off))
        w, lo, hi = _node(kids, 0, base)
        inner.append(w)
        kids_root.append((lo, hi, 0xFF))
    root, _, _ = _node(kids_root, 1, 0)
    return np.stack([root] + inner), np.asarray(recs, np.float32)


def _rays(seed, n):
    rays = scenes.random_rays(seed, n)
    # axis-parallel directions exercise the guarded 1/d of a zero component
    k = n // 8
    d = np.zeros((k, 3), np.float32)
    d[np.arange(k), np.arange(k) % 3] = np.where(np.arange(k) % 2, 1.0, -1.0)
    rays["dir"][:k] = d
    return rays


def test_walk_matches_brute_force_on_hand_built_tree():
    rng = np.random.default_rng(17)
    c = rng.uniform(-8, 8, (180, 1, 3)).astype(np.float32)
    tris = (c + rng.uniform(-2.5, 2.5, (180, 3, 3)).astype(np.float32)).reshape(-1, 9)
    nodes, recs = hand_built_tree(tris)
    rays = _rays(3, 4000)
    rays["org"] *= np.float32(0.12)  # start inside the 10-unit cloud
    hits, cnt = O.walk_bvh8(nodes, recs, rays)
    ref = O.brute_closest(tris, rays)
    assert (ref["prim"] >= 0).mean() > 0.3
    assert np.array_equal(hits["prim"], ref["prim"])
    for f in ("t", "u", "v"):
        assert np.array_equal(hits[f].view(np.uint32), ref[f].view(np.uint32)), f
    occ, cnt_any = O.walk_bvh8(nodes, recs, rays, any_hit=True)
    assert np.array_equal(occ, O.brute_any(tris, rays))
    assert (cnt[:, 0] >= 1).all() and (cnt_any[:, 0] >= 1).all()  # every walk visits the root
    # one round per node visit or two: the same hits either way
    hits1, cnt1 = O.walk_bvh8(nodes, recs, rays, niters=1)
    assert np.array_equal(hits1.view(np.uint8), hits.view(np.uint8))


def test_walk_rejects_indices_past_the_arrays():
    rng = np.random.default_rng(5)
    tris = rng.uniform(-1, 1, (40, 9)).astype(np.float32)
    nodes, recs = hand_built_tree(tris)
    rays = _rays(9, 500)
    rays["org"] *= np.float32(0.01)
    nodes[0, 4] = 1000  # root's first child past the node array
    with pytest.raises(ValueError):
        O.walk_bvh8(nodes, recs, rays)


@pytest.mark.parametrize("path", sorted(GOLD.glob("bvh8_walk_*.npz")), ids=lambda p: p.stem)
def test_walk_reproduces_the_kernel(path):
    from rtb200.scenes import HIT_DTYPE

    g = np.load(path)
    rays = np.ascontiguousarray(g["rays"]).view(RAY_DTYPE).reshape(-1)
    shadow = np.ascontiguousarray(g["shadow"]).view(RAY_DTYPE).reshape(-1)
    # the walk shape of the kernel that wrote the fixture
    shape = dict(niters=int(g["niters"]), sets=int(g["sets"]))
    assert (shape["niters"], shape["sets"]) == (O.KERNEL_NITERS, O.KERNEL_SETS), "fixture of another kernel"
    hits, cnt = O.walk_bvh8(g["nodes"], g["recs"], rays, **shape)
    ref = np.ascontiguousarray(g["hits"]).view(HIT_DTYPE).reshape(-1)
    assert (ref["prim"] >= 0).any()
    assert np.array_equal(hits.view(np.uint8), ref.view(np.uint8))  # t, primitive, u, v bit for bit
    assert np.array_equal(cnt, g["counts_closest"])  # node visits and triangle tests, every ray
    occ, cnt_any = O.walk_bvh8(g["nodes"], g["recs"], shadow, any_hit=True, **shape)
    assert 0 < occ.sum() < occ.size
    assert np.array_equal(occ, g["occ"])
    assert np.array_equal(cnt_any, g["counts_any"])
    # the algorithmic bytes per ray bench.py charges, from the oracle's counts
    per_ray = 32 + 16 + cnt[:, 0].mean() * 80 + cnt[:, 1].mean() * 36
    assert per_ray > 48


def _slot_boxes(node):
    """Decoded child boxes of one 8-wide node (float64): lo, hi (8, 3)."""
    p = node[0:3].view(np.float32).astype(np.float64)
    e = int(node[3])
    scale = np.array([math.ldexp(1.0, ((e >> (8 * a)) & 0xFF) - 127) if (e >> (8 * a)) & 0xFF else 0.0
                      for a in range(3)])
    lo, hi = np.zeros((8, 3)), np.zeros((8, 3))
    for a in range(3):
        w = [int(x) for x in node[8 + 4 * a: 12 + 4 * a]]
        for s in range(8):
            ql = (w[s >> 2] >> (8 * (s & 3))) & 0xFF
            qh = (w[2 + (s >> 2)] >> (8 * (s & 3))) & 0xFF
            lo[s, a], hi[s, a] = p[a] + ql * scale[a], p[a] + qh * scale[a]
    return lo, hi


@pytest.mark.parametrize("path", sorted(GOLD.glob("bvh8_walk_*.npz")), ids=lambda p: p.stem)
def test_quantised_boxes_hold_their_triangles(path):
    """The builder's 8-bit child boxes are rounded outward: every triangle
    reachable through a slot lies inside that slot's decoded box (the tree
    the kernel walked, as written on the GPU)."""
    g = np.load(path)
    nodes, recs = g["nodes"], g["recs"].astype(np.float64)
    v0 = recs[:, 0:3]
    verts = np.stack([v0, v0 + recs[:, 4:7], v0 + recs[:, 8:11]], 1)  # the triangle the kernel tests
    memo = {}

    def slot_records(ni):
        node = nodes[ni]
        imask, child_base, tri_base = int(node[3]) >> 24, int(node[4]), int(node[5])
        per_slot = []
        for s in range(8):
            meta = (int(node[6 + (s >> 2)]) >> (8 * (s & 3))) & 0xFF
            if (imask >> s) & 1:
                c = child_base + bin(imask & ((1 << s) - 1)).count("1")
                per_slot.append(subtree(c))
            else:
                per_slot.append(np.arange(tri_base + (meta & 31), tri_base + (meta & 31) + (meta >> 5)))
        return per_slot

    def subtree(ni):
        if ni not in memo:
            memo[ni] = np.concatenate(slot_records(ni))
        return memo[ni]

    checked = 0
    for ni in range(nodes.shape[0]):
        lo, hi = _slot_boxes(nodes[ni])
        for s, r in enumerate(slot_records(ni)):
            if r.size == 0:
                continue
            v = verts[r].reshape(-1, 3)
            tol = 1e-6 * (np.abs(v).max() + 1.0)  # the stored edges are rounded differences
            assert (v >= lo[s] - tol).all() and (v <= hi[s] + tol).all(), (ni, s)
            checked += 1
    assert sorted(subtree(0).tolist()) == list(range(recs.shape[0]))  # every record under the root once
    assert checked > nodes.shape[0]
